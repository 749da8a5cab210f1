// Serving engine: takes subspace requests (S = Psi^T Psi, Hs = Psi^T H Psi,
// then Psi' = Psi Q) as they arrive, admits them by free HBM, keeps each
// request's Psi resident across its three steps, and overlaps requests on
// the device.
//
// Native FP64 uses continuous batching: each engine step gathers the ready
// steps of all admitted requests -- S and Hs of requests whose inputs are on
// the device, rotations of requests whose S and Hs are done -- into one
// grouped persistent Stream-K launch (skg_batch.h) on a single compute
// stream, with up to two launches in flight. Grouped launches never overlap
// each other, so their CTAs never wait on CTAs that cannot become resident;
// input generation and layout conversion overlap them on a second stream.
// The Ozaki path runs each admitted request's whole sequence on one of a few
// slot streams (its kernels have no inter-CTA waits), with the slots'
// scratch reserved up front for the largest request of the trace.
//
// Memory: request data lives in one device arena of the admission budget
// minus the engine's fixed scratch; a request is admitted, in arrival order,
// when a contiguous block for all its buffers is free (first fit with
// coalescing). Freed blocks are reused after the host has seen the
// request's last kernel complete.
//
// The scheduler is written against an executor interface: the GPU executor
// runs the kernels and times completions with CUDA events; the simulated
// executor replaces them with a throughput model on a virtual clock, so the
// admission and batching logic runs without a GPU.
//
// The reference has no serving layer: its drivers run one kernel on one
// problem at a time (gemm_opt.cpp:397-425 and :511-557, syrk_crsp.cpp:425-528).
// The synthetic requests follow the DFT subspace shapes of those drivers.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "skg_batch.h"
#include "skg_ozaki.h"
#include "skg_runtime.h"

namespace skg {

// ------------------------------------------------------- synthetic inputs
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014).
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(uint64_t h) {  // uniform in (0, 1)
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// x[i] = scale * N(0,1), a pure function of (seed, i): Box-Muller on two
// counter-based uniforms per pair of outputs.
__global__ void gen_normal_kernel(double* __restrict__ x, int64_t n, uint64_t seed,
                                  double scale) {
  const int64_t pairs = (n + 1) / 2;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < pairs;
       p += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = mix64(seed ^ mix64((uint64_t)p));
    const double u1 = u01(h), u2 = u01(mix64(h ^ 0xD1B54A32D192ED03ull));
    const double r = sqrt(-2.0 * log(u1)) * scale;
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    const int64_t i = 2 * p;
    x[i] = r * cs;
    if (i + 1 < n) x[i + 1] = r * sn;
  }
}

__global__ void gen_uniform_kernel(double* __restrict__ x, int64_t n, uint64_t seed, double lo,
                                   double hi) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = lo + (hi - lo) * u01(mix64(seed ^ mix64((uint64_t)i)));
}

int launch_gen_normal(double* x, int64_t n, uint64_t seed, double scale, int sms,
                      cudaStream_t s) {
  if (n <= 0) return SKGEMM_OK;
  const int64_t blocks = std::min<int64_t>((int64_t)sms * 8, ((n + 1) / 2 + 255) / 256);
  gen_normal_kernel<<<(unsigned)blocks, 256, 0, s>>>(x, n, seed, scale);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int launch_gen_uniform(double* x, int64_t n, uint64_t seed, double lo, double hi, int sms,
                       cudaStream_t s) {
  if (n <= 0) return SKGEMM_OK;
  const int64_t blocks = std::min<int64_t>((int64_t)sms * 8, (n + 255) / 256);
  gen_uniform_kernel<<<(unsigned)blocks, 256, 0, s>>>(x, n, seed, lo, hi);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

}  // namespace

namespace serve {

constexpr size_t kAlign = 512;
inline size_t al(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Buffers of one request, in arena order.
struct Layout {
  size_t psi16, h32, grid, out, S, Hs, Q, total;
};

Layout layout_of(int64_t Ng, int64_t nb) {
  Layout L;
  const int64_t nb32 = (nb + 31) / 32 * 32;
  L.psi16 = 0;
  L.h32 = L.psi16 + al((size_t)Ng * nb * 8);
  L.grid = L.h32 + al((size_t)Ng * nb32 * 8);
  L.out = L.grid + al((size_t)Ng * nb * 8);
  L.S = L.out + al((size_t)Ng * nb * 8);
  L.Hs = L.S + al((size_t)nb * nb * 8);
  L.Q = L.Hs + al((size_t)nb * nb * 8);
  L.total = L.Q + al((size_t)nb * nb * 8);
  return L;
}

// First-fit arena with coalescing (host bookkeeping of device offsets).
class Arena {
 public:
  explicit Arena(size_t cap) : cap_(cap) {
    if (cap) free_[0] = cap;
  }
  bool alloc(size_t bytes, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, noff = it->first + bytes;
        free_.erase(it);
        if (rest) free_[noff] = rest;
        used_ += bytes;
        peak_ = std::max(peak_, used_);
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t capacity() const { return cap_; }
  size_t peak() const { return peak_; }
  size_t used() const { return used_; }

 private:
  size_t cap_, used_ = 0, peak_ = 0;
  std::map<size_t, size_t> free_;
};

enum State { kWait, kGen, kRun1, kReady2, kRun2, kDone };

struct Req {
  int idx = 0;
  int64_t Ng = 0, nb = 0;
  double arrival = 0.0;
  uint64_t seed = 0;
  Layout lay{};
  size_t off = 0;
  int state = kWait;
  int slot = -1;
  double admit = 0.0, done = 0.0;
  double flop = 0.0;
  // executor-owned
  cudaEvent_t gen_ev = nullptr, done_ev = nullptr;
  double sim_gen_done = 0.0, sim_done = 0.0;
};

struct Batch {
  std::vector<int> s1, s2;  // requests whose S+Hs / rotation run in this launch
  double flop = 0.0;
  int problems = 0;
  cudaEvent_t ev = nullptr;
  double sim_done = 0.0;
};

// FLOPs of a request: S = Psi^T Psi counted M^2 K (the reference's SYRK count,
// syrk_crsp.cpp:456-457), Hs 2 M N K, rotation 2 Nd nb^2 (trp_3d_test.cpp:195).
inline double request_flop(int64_t Ng, int64_t nb) {
  const double n2 = (double)nb * (double)nb, g = (double)Ng;
  return n2 * g + 2.0 * n2 * g + 2.0 * g * n2;
}

struct Exec {
  virtual ~Exec() {}
  virtual double now() = 0;
  virtual int gen(Req& r) = 0;
  virtual bool gen_ready(Req& r) = 0;
  virtual int launch(Batch& b, std::vector<Req>& R) = 0;
  virtual bool batch_ready(Batch& b) = 0;
  virtual double batch_time(Batch& b) = 0;
  virtual int run_ozaki(Req& r) = 0;
  virtual bool req_ready(Req& r) = 0;
  virtual double req_time(Req& r) = 0;
  virtual int finish(Req& r, const skgemm_serve_request_t& io) = 0;
  virtual void idle(double next_arrival) = 0;
  // True when idle() could not move time forward (simulation with nothing
  // pending: a scheduler bug, reported instead of spinning).
  virtual bool stalled(double before) { (void)before; return false; }
  virtual int error() = 0;
};

// ------------------------------------------------------------ GPU executor
struct GpuExec : Exec {
  DeviceState* dev = nullptr;
  int precision = SKGEMM_PREC_NATIVE, slices = 0;
  char* arena = nullptr;
  cudaStream_t comp = nullptr, gens = nullptr;
  std::vector<cudaStream_t> slots;
  GroupRing* ring = nullptr;
  cudaEvent_t t0 = nullptr;
  std::chrono::steady_clock::time_point h0;
  std::vector<cudaEvent_t> pool;  // recycled timing events
  int status = SKGEMM_OK;

  cudaEvent_t ev() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
  }
  void give(cudaEvent_t& e) {
    if (e) pool.push_back(e);
    e = nullptr;
  }
  double* p(const Req& r, size_t o) { return (double*)(arena + r.off + o); }

  double now() override {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - h0).count();
  }
  int fill(Req& r, cudaStream_t s) {
    int st;
    const int64_t nb32 = (r.nb + 31) / 32 * 32;
    const double sc = 1.0 / std::sqrt((double)r.Ng);
    if ((st = launch_gen_normal(p(r, r.lay.psi16), r.Ng * r.nb, r.seed * 4 + 0, sc,
                                dev->num_sms, s)))
      return st;
    if ((st = launch_gen_normal(p(r, r.lay.h32), r.Ng * nb32, r.seed * 4 + 1, sc, dev->num_sms,
                                s)))
      return st;
    if ((st = launch_gen_uniform(p(r, r.lay.Q), r.nb * r.nb, r.seed * 4 + 2, -1.0, 1.0,
                                 dev->num_sms, s)))
      return st;
    // The rotation reads Psi grid-packed; the subspace products read it band-packed.
    return launch_band_to_grid(r.Ng, r.nb, p(r, r.lay.psi16), p(r, r.lay.grid), s);
  }
  int gen(Req& r) override {
    int st = fill(r, gens);
    if (st) return st;
    if (!(r.gen_ev = ev())) return fail(SKGEMM_ERR_CUDA, "cudaEventCreate");
    SKG_CUDA(cudaEventRecord(r.gen_ev, gens));
    return SKGEMM_OK;
  }
  bool gen_ready(Req& r) override { return cudaEventQuery(r.gen_ev) == cudaSuccess; }
  int launch(Batch& b, std::vector<Req>& R) override {
    std::vector<Fp64Problem> probs;
    for (int i : b.s1) {
      Req& r = R[i];
      probs.push_back(syrk_problem(r.Ng, r.nb, p(r, r.lay.psi16), p(r, r.lay.S), r.nb, 1.0, 0.0));
      probs.push_back(gemm_packed_problem(r.nb, r.nb, r.Ng, p(r, r.lay.psi16), p(r, r.lay.h32),
                                          p(r, r.lay.Hs), r.nb, 1.0, 0.0));
      give(r.gen_ev);
    }
    for (int i : b.s2) {
      Req& r = R[i];
      probs.push_back(rot_problem(r.Ng, r.nb, p(r, r.lay.grid), p(r, r.lay.Q), p(r, r.lay.out)));
    }
    int st = group_ring_submit(ring, probs, comp, nullptr);
    if (st) return st;
    if (!(b.ev = ev())) return fail(SKGEMM_ERR_CUDA, "cudaEventCreate");
    SKG_CUDA(cudaEventRecord(b.ev, comp));
    return SKGEMM_OK;
  }
  bool batch_ready(Batch& b) override { return cudaEventQuery(b.ev) == cudaSuccess; }
  double batch_time(Batch& b) override {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, b.ev);
    give(b.ev);
    return ms * 1e-3;
  }
  int run_ozaki(Req& r) override {
    cudaStream_t s = slots[r.slot];
    int st = fill(r, s);
    if (st) return st;
    skgemm_options_t o;
    memset(&o, 0, sizeof(o));
    o.precision = SKGEMM_PREC_OZAKI_I8;
    o.slices = slices;
    // S and Hs from one split of Psi (the subspace pair).
    if ((st = skgemm_dsubspace_packed_dev(r.Ng, r.nb, p(r, r.lay.psi16), p(r, r.lay.h32),
                                          p(r, r.lay.S), r.nb, p(r, r.lay.Hs), r.nb, &o, s)))
      return st;
    if ((st = skgemm_drot_dev_opt(r.Ng, r.nb, p(r, r.lay.grid), p(r, r.lay.Q), p(r, r.lay.out),
                                  &o, s)))
      return st;
    if (!(r.done_ev = ev())) return fail(SKGEMM_ERR_CUDA, "cudaEventCreate");
    SKG_CUDA(cudaEventRecord(r.done_ev, s));
    return SKGEMM_OK;
  }
  bool req_ready(Req& r) override { return cudaEventQuery(r.done_ev) == cudaSuccess; }
  double req_time(Req& r) override {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, r.done_ev);
    give(r.done_ev);
    return ms * 1e-3;
  }
  int finish(Req& r, const skgemm_serve_request_t& io) override {
    const size_t n2 = (size_t)r.nb * r.nb * 8, big = (size_t)r.Ng * r.nb * 8;
    const int64_t nb32 = (r.nb + 31) / 32 * 32;
    struct {
      double* dst;
      size_t off, bytes;
    } cp[6] = {{io.S_out, r.lay.S, n2},
               {io.Hs_out, r.lay.Hs, n2},
               {io.Psi_out, r.lay.out, big},
               {io.Psi_in_out, r.lay.psi16, big},
               {io.HPsi_in_out, r.lay.h32, (size_t)r.Ng * nb32 * 8},
               {io.Q_in_out, r.lay.Q, n2}};
    for (auto& c : cp)
      if (c.dst) SKG_CUDA(cudaMemcpy(c.dst, arena + r.off + c.off, c.bytes, cudaMemcpyDeviceToHost));
    return SKGEMM_OK;
  }
  void idle(double) override { std::this_thread::sleep_for(std::chrono::microseconds(20)); }
  int error() override {
    int st = ring ? group_ring_error(ring) : SKGEMM_OK;
    if (st) return st;
    for (cudaStream_t s : slots)
      if ((st = skgemm_stream_status(s))) return st;
    return SKGEMM_OK;
  }
  ~GpuExec() override {
    cudaDeviceSynchronize();
    for (cudaStream_t s : slots) skgemm_stream_release(s);
    if (ring) group_ring_destroy(ring);
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
    if (t0) cudaEventDestroy(t0);
    if (arena) cudaFree(arena);
    if (comp) cudaStreamDestroy(comp);
    if (gens) cudaStreamDestroy(gens);
    for (cudaStream_t s : slots) cudaStreamDestroy(s);
  }
};

// ------------------------------------------------------- simulated executor
// Virtual clock; the compute stream runs grouped launches back to back at
// `tflops` on the issued MACs' useful share; generation streams at `gen_gbs`;
// Ozaki slots share the device at `oz_tflops`.
struct SimExec : Exec {
  double t = 0.0, comp_free = 0.0, gen_free = 0.0, dev_free = 0.0;
  double tflops = 30.0, oz_tflops = 45.0, gen_gbs = 3000.0;
  std::vector<double> pending;  // completion times still ahead

  double now() override { return t; }
  int gen(Req& r) override {
    const double bytes = (double)r.lay.total;
    gen_free = std::max(t, gen_free) + bytes / (gen_gbs * 1e9);
    r.sim_gen_done = gen_free;
    pending.push_back(gen_free);
    return SKGEMM_OK;
  }
  bool gen_ready(Req& r) override { return r.sim_gen_done <= t; }
  int launch(Batch& b, std::vector<Req>& R) override {
    (void)R;
    comp_free = std::max(t, comp_free) + b.flop / (tflops * 1e12);
    b.sim_done = comp_free;
    pending.push_back(comp_free);
    return SKGEMM_OK;
  }
  bool batch_ready(Batch& b) override { return b.sim_done <= t; }
  double batch_time(Batch& b) override { return b.sim_done; }
  int run_ozaki(Req& r) override {
    const double g = std::max(t, gen_free) + (double)r.lay.total / (gen_gbs * 1e9);
    gen_free = g;
    dev_free = std::max(g, dev_free) + r.flop / (oz_tflops * 1e12);
    r.sim_done = dev_free;
    pending.push_back(dev_free);
    return SKGEMM_OK;
  }
  bool req_ready(Req& r) override { return r.sim_done <= t; }
  double req_time(Req& r) override { return r.sim_done; }
  int finish(Req&, const skgemm_serve_request_t&) override { return SKGEMM_OK; }
  void idle(double next_arrival) override {
    double nx = next_arrival;
    for (double x : pending)
      if (x > t) nx = std::min(nx, x);
    pending.erase(std::remove_if(pending.begin(), pending.end(), [&](double x) { return x <= nx; }),
                  pending.end());
    if (nx > t && nx < 1e300) t = nx;
  }
  bool stalled(double before) override { return t <= before; }
  int error() override { return SKGEMM_OK; }
};

// ---------------------------------------------------------------- scheduler
int schedule(skgemm_serve_request_t* io, int n, skgemm_serve_options_t& o, Exec& ex,
             Arena& arena, int nslots) {
  const bool native = (o.precision == SKGEMM_PREC_NATIVE);
  std::vector<Req> R(n);
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) {
    Req& r = R[i];
    r.idx = i;
    r.Ng = io[i].Ng;
    r.nb = io[i].nb;
    r.arrival = o.realtime ? io[i].arrival_s : 0.0;
    r.seed = io[i].seed;
    r.lay = layout_of(r.Ng, r.nb);
    r.flop = request_flop(r.Ng, r.nb);
    order[i] = i;
    if (r.lay.total > arena.capacity()) {
      char buf[200];
      snprintf(buf, sizeof(buf),
               "serve: request %d (Ng %lld, nb %lld) needs %.2f GB, more than the %.2f GB the "
               "budget leaves for request data",
               i, (long long)r.Ng, (long long)r.nb, r.lay.total / 1e9, arena.capacity() / 1e9);
      return fail(SKGEMM_ERR_OOM, buf);
    }
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return R[a].arrival < R[b].arrival; });
  const double cap = (o.max_batch_tflop > 0 ? o.max_batch_tflop : 2.0) * 1e12;
  const int max_inflight = o.max_inflight > 0 ? o.max_inflight : 64;
  std::deque<int> queue, gen_wait, ready2;
  std::deque<Batch> flight;
  std::vector<int> slot_req(nslots, -1);
  int next = 0, done = 0, inflight = 0, st;
  int batches = 0;
  double batch_problems = 0.0, makespan = 0.0, flop = 0.0;
  double last_progress = ex.now();
  constexpr double kStallSeconds = 120.0;

  auto complete = [&](Req& r, double t) -> int {
    r.done = t;
    r.state = kDone;
    int s2 = ex.finish(r, io[r.idx]);
    arena.release(r.off, r.lay.total);
    --inflight;
    ++done;
    makespan = std::max(makespan, t);
    flop += r.flop;
    io[r.idx].admit_s = r.admit;
    io[r.idx].done_s = r.done;
    return s2;
  };

  while (done < n) {
    const double t = ex.now();
    bool progressed = false;
    while (next < n && R[order[next]].arrival <= t) {
      queue.push_back(order[next++]);
      progressed = true;
    }
    // Completions.
    if (native) {
      while (!flight.empty() && ex.batch_ready(flight.front())) {
        Batch b = flight.front();
        flight.pop_front();
        const double bt = ex.batch_time(b);
        for (int i : b.s1) {
          R[i].state = kReady2;
          ready2.push_back(i);
        }
        for (int i : b.s2)
          if ((st = complete(R[i], bt))) return st;
        progressed = true;
      }
    } else {
      for (int k = 0; k < nslots; ++k) {
        const int i = slot_req[k];
        if (i >= 0 && ex.req_ready(R[i])) {
          slot_req[k] = -1;
          if ((st = complete(R[i], ex.req_time(R[i])))) return st;
          progressed = true;
        }
      }
    }
    // Admission while a slot and a contiguous block are free: the request at
    // the head of the queue (FIFO), or the waiting request with the least
    // work, its work discounted by its wait (SMALLEST: small requests stop
    // queueing behind large ones; the discount bounds any request's wait).
    while (!queue.empty()) {
      auto pick = queue.begin();
      if (o.policy == SKGEMM_SERVE_SMALLEST) {
        const double tau = o.aging_s > 0 ? o.aging_s : 1.0;
        double best = 1e300;
        for (auto it = queue.begin(); it != queue.end(); ++it) {
          const Req& c = R[*it];
          const double key = c.flop / (1.0 + std::max(0.0, t - c.arrival) / tau);
          if (key < best) {
            best = key;
            pick = it;
          }
        }
      } else if (o.policy == SKGEMM_SERVE_RATIO) {
        // Response ratio (wait + service) / service = 1 + wait / service, and
        // service is proportional to work: the largest wait / work wins.
        double best = -1.0, best_flop = 1e300;
        for (auto it = queue.begin(); it != queue.end(); ++it) {
          const Req& c = R[*it];
          const double key = std::max(0.0, t - c.arrival) / std::max(c.flop, 1.0);
          if (key > best || (key == best && c.flop < best_flop)) {
            best = key;
            best_flop = c.flop;
            pick = it;
          }
        }
      }
      Req& r = R[*pick];
      int k = -1;
      if (native) {
        if (inflight >= max_inflight) break;
      } else {
        for (int j = 0; j < nslots && k < 0; ++j)
          if (slot_req[j] < 0) k = j;
        if (k < 0) break;
      }
      if (!arena.alloc(r.lay.total, &r.off)) break;
      queue.erase(pick);
      ++inflight;
      r.admit = t;
      if (native) {
        r.state = kGen;
        if ((st = ex.gen(r))) return st;
        gen_wait.push_back(r.idx);
      } else {
        r.slot = k;
        slot_req[k] = r.idx;
        r.state = kRun1;
        if ((st = ex.run_ozaki(r))) return st;
      }
      progressed = true;
    }
    // Continuous batching: one grouped launch of every ready step, oldest
    // first, up to the work cap; at most two launches in flight.
    if (native && flight.size() < 2) {
      Batch b;
      while (!ready2.empty() && (b.flop < cap || b.problems == 0)) {
        Req& r = R[ready2.front()];
        ready2.pop_front();
        r.state = kRun2;
        b.s2.push_back(r.idx);
        b.flop += 2.0 * (double)r.Ng * r.nb * r.nb;
        b.problems += 1;
      }
      while (!gen_wait.empty() && (b.flop < cap || b.problems == 0) &&
             ex.gen_ready(R[gen_wait.front()])) {
        Req& r = R[gen_wait.front()];
        gen_wait.pop_front();
        r.state = kRun1;
        b.s1.push_back(r.idx);
        b.flop += 3.0 * (double)r.Ng * r.nb * r.nb;
        b.problems += 2;
      }
      if (b.problems > 0) {
        if ((st = ex.launch(b, R))) return st;
        flight.push_back(b);
        ++batches;
        batch_problems += b.problems;
        progressed = true;
      }
    }
    if (progressed) {
      last_progress = ex.now();
    } else {
      if (ex.now() - last_progress > kStallSeconds)
        return fail(SKGEMM_ERR_DEVICE_TIMEOUT, "serve: no request made progress for 120 s");
      const double before = ex.now();
      ex.idle(next < n ? R[order[next]].arrival : 1e300);
      if (ex.stalled(before)) return fail(SKGEMM_ERR_UNSUPPORTED, "serve: scheduler has no event to wait for");
    }
  }
  o.makespan_s = makespan;
  o.flop = flop;
  o.batches = batches;
  o.mean_batch_problems = batches ? batch_problems / batches : 0.0;
  o.peak_admitted_bytes = (double)arena.peak();
  return ex.error();
}

}  // namespace serve

int serve_run(skgemm_serve_request_t* io, int n, skgemm_serve_options_t* opts, bool simulate) {
  using namespace serve;
  if (!opts) return fail(SKGEMM_ERR_INVALID_ARG, "null serve options");
  if (n < 0 || (n > 0 && !io)) return fail(SKGEMM_ERR_INVALID_ARG, "bad request array");
  skgemm_serve_options_t& o = *opts;
  if (o.precision != SKGEMM_PREC_NATIVE && o.precision != SKGEMM_PREC_OZAKI_I8)
    return fail(SKGEMM_ERR_INVALID_ARG, "serve: unknown precision");
  if (o.policy != SKGEMM_SERVE_FIFO && o.policy != SKGEMM_SERVE_SMALLEST &&
      o.policy != SKGEMM_SERVE_RATIO)
    return fail(SKGEMM_ERR_INVALID_ARG, "serve: unknown admission policy");
  if (o.aging_s < 0) return fail(SKGEMM_ERR_INVALID_ARG, "serve: aging_s must be >= 0");
  int64_t max_ng = 0, max_nb = 0;
  for (int i = 0; i < n; ++i) {
    if (io[i].Ng <= 0 || io[i].nb <= 0 || io[i].Ng % 16 || io[i].nb % 16)
      return fail(SKGEMM_ERR_INVALID_ARG,
                  "serve: Ng and nb must be positive multiples of 16 (packed layouts)");
    if (o.precision == SKGEMM_PREC_OZAKI_I8 && io[i].nb > 2048)
      return fail(SKGEMM_ERR_UNSUPPORTED, "serve: Ozaki rotation supports nb <= 2048");
    max_ng = std::max(max_ng, io[i].Ng);
    max_nb = std::max(max_nb, io[i].nb);
  }
  const double budget = o.hbm_budget_bytes > 0 ? o.hbm_budget_bytes : 150e9;
  const int nslots = o.precision == SKGEMM_PREC_NATIVE ? 0 : (o.ozaki_streams > 0 ? o.ozaki_streams : 2);
  o.makespan_s = o.flop = o.mean_batch_problems = o.peak_admitted_bytes = o.scratch_bytes = 0.0;
  o.batches = 0;
  if (n == 0) return SKGEMM_OK;

  if (simulate) {
    SimExec ex;
    if (o.sim_native_tflops > 0) ex.tflops = o.sim_native_tflops;
    if (o.sim_ozaki_tflops > 0) ex.oz_tflops = o.sim_ozaki_tflops;
    if (o.sim_gen_gbs > 0) ex.gen_gbs = o.sim_gen_gbs;
    Arena arena((size_t)budget);
    return schedule(io, n, o, ex, arena, nslots);
  }

  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  std::unique_ptr<GpuExec> ex(new GpuExec());
  ex->dev = dev;
  ex->precision = o.precision;
  ex->slices = o.slices;
  SKG_CUDA(cudaStreamCreateWithFlags(&ex->comp, cudaStreamNonBlocking));
  SKG_CUDA(cudaStreamCreateWithFlags(&ex->gens, cudaStreamNonBlocking));
  double scratch = 0.0;
  if (o.precision == SKGEMM_PREC_NATIVE) {
    const int max_inflight = o.max_inflight > 0 ? o.max_inflight : 64;
    ex->ring = group_ring_create(dev, 3);
    if ((st = group_ring_reserve(ex->ring, 3 * max_inflight))) return st;
    scratch = 3.0 * 148 * 128 * 128 * 8;
  } else {
    for (int k = 0; k < nslots; ++k) {
      cudaStream_t s;
      SKG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      ex->slots.push_back(s);
      if ((st = ozaki_reserve(dev, s, max_ng, max_nb, o.slices))) return st;
      scratch += (double)ozaki_stream_bytes(dev, s);
    }
  }
  o.scratch_bytes = scratch;
  if (scratch >= budget) return fail(SKGEMM_ERR_OOM, "serve: scratch exceeds the HBM budget");
  const size_t arena_bytes = (size_t)(budget - scratch) / 4096 * 4096;
  SKG_CUDA(cudaMalloc(&ex->arena, arena_bytes));
  Arena arena(arena_bytes);
  SKG_CUDA(cudaEventCreate(&ex->t0));
  SKG_CUDA(cudaDeviceSynchronize());
  SKG_CUDA(cudaEventRecord(ex->t0, ex->comp));
  ex->h0 = std::chrono::steady_clock::now();
  st = serve::schedule(io, n, o, *ex, arena, nslots);
  cudaDeviceSynchronize();
  return st;
}

}  // namespace skg

using namespace skg;

#define SKG_EXPORT extern "C" __attribute__((visibility("default")))

SKG_EXPORT int skgemm_serve_run(skgemm_serve_request_t* reqs, int n,
                                skgemm_serve_options_t* opts) {
  NvtxRange nvtx_(__func__);
  return serve_run(reqs, n, opts, false);
}

SKG_EXPORT int skgemm_serve_simulate(skgemm_serve_request_t* reqs, int n,
                                     skgemm_serve_options_t* opts) {
  return serve_run(reqs, n, opts, true);
}
