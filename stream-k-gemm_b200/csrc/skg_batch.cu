// Batched path: many independent GEMM / SYRK / rotation problems of uneven
// sizes in one grouped persistent Stream-K launch, a plan that autotunes the
// tile shape, problem order and grid, and records the launch into a CUDA
// graph.
//
// The reference has no batched entry point: its CheFSI driver calls
// sme_syrk<double>::compute (include/sme_syrk.hpp:137) and
// gemm<double>::compute_packed (gemm_opt.cpp:314) once per k-point / spin
// block. Each item here keeps the contract of the matching single-problem
// call (skgemm_dsyrk_packed_dev, skgemm_dgemm_packed_dev, skgemm_drot_dev).
//
// Schedule: problem p contributes num_tiles(p) * ceil(K(p)/16) MAC-loop
// iterations; the iterations of all problems are concatenated in the plan's
// problem order and split evenly over the persistent CTAs (Fp64Group). Tuning
// candidates: tile 128x128 (1 CTA/SM) or 64x64 (2 CTAs/SM: less padding waste
// on small state counts, same DMMA fragment code), problem order as given or
// most-work-first, and the grid. The cost model is the useful/issued MAC
// ratio of the tiles; tuning times each candidate with CUDA events on the
// items' own buffers and keeps the fastest (cached per batch signature).
//
// Precision per problem: a plan may run some problems through the Ozaki
// split (skg_ozaki.cu) instead of the grouped FP64 launch. Under
// SKGEMM_PREC_AUTO the cost model compares each problem's share of the
// grouped launch (issued MACs at the measured DMMA rate) with the Ozaki
// kernels' estimate (ozaki_time_estimate) and picks Ozaki where it is below
// 0.8 of native; tuning also times the all-native assignment and keeps the
// faster. A SYRK and a GEMM of the same band-packed operand (S = Psi^T Psi and
// Hs = Psi^T HPsi of one k-point) both sent to the Ozaki split run as one
// subspace pair that converts Psi once (ozaki_subspace), and the cost model
// prices them as a pair. Ozaki problems run one after another on a stream the plan owns, so
// their scratch buffers (which the captured graph references) belong to the
// plan and cannot be regrown by unrelated calls.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "skg_batch.h"
#include "skg_fp64_types.h"
#include "skg_ozaki.h"
#include "skg_runtime.h"

namespace skg {

namespace {

struct Geom {
  int tiles_m = 0, tiles_n = 0, num_tiles = 0, ipt = 0;
  int64_t iters = 0;
  double useful = 0.0, issued = 0.0;  // MACs
};

// Validates one item and builds its problem descriptor (zero-size items are
// valid and produce no iterations).
int item_problem(const skgemm_batch_item_t& it, Fp64Problem* p) {
  if (it.M < 0 || it.N < 0 || it.K < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative dimension");
  switch (it.op) {
    case SKGEMM_OP_GEMM_PACKED:
      if (it.ldd < it.N) return fail(SKGEMM_ERR_INVALID_ARG, "batch item: ldd < N");
      *p = gemm_packed_problem(it.M, it.N, it.K, it.A, it.B, it.D, it.ldd, it.alpha, it.beta);
      break;
    case SKGEMM_OP_SYRK_PACKED:
      if (it.ldd < it.M) return fail(SKGEMM_ERR_INVALID_ARG, "batch item: ldc < M");
      *p = syrk_problem(it.K, it.M, it.A, it.D, it.ldd, it.alpha, it.beta);
      break;
    case SKGEMM_OP_ROT:
      if (it.M % 16 || it.N % 16)
        return fail(SKGEMM_ERR_INVALID_ARG,
                    "batch item: rotation layouts need Nd and nb multiples of 16");
      *p = rot_problem(it.M, it.N, it.A, it.B, it.D);
      break;
    default:
      return fail(SKGEMM_ERR_INVALID_ARG, "batch item: unknown op");
  }
  if (p->K > (int64_t)INT32_MAX - kBK || p->M > ((int64_t)1 << 31) || p->N > ((int64_t)1 << 31))
    return fail(SKGEMM_ERR_INVALID_ARG, "batch item: dimension too large");
  if (p->M > 0 && p->N > 0) {
    if (!p->D) return fail(SKGEMM_ERR_INVALID_ARG, "batch item: null output pointer");
    if (p->K > 0 && (!p->a.ptr || !p->b.ptr))
      return fail(SKGEMM_ERR_INVALID_ARG, "batch item: null operand pointer");
  }
  return SKGEMM_OK;
}

Geom geom_of(const Fp64Problem& p, int BM, int BN) {
  Geom g;
  if (p.M == 0 || p.N == 0 || p.K == 0) return g;
  g.tiles_m = (int)((p.M + BM - 1) / BM);
  g.tiles_n = (int)((p.N + BN - 1) / BN);
  if (p.tile_order == kTilesUpper) {
    // Upper-triangle tiles: tile (tm, tn) with tm*BM <= tn*BN + BN - 1. For
    // square tiles that is tm <= tn.
    g.num_tiles = g.tiles_n * (g.tiles_n + 1) / 2;
    g.useful = (double)p.M * (double)(p.M + 1) / 2.0 * (double)p.K;
  } else {
    g.num_tiles = g.tiles_m * g.tiles_n;
    g.useful = (double)p.M * (double)p.N * (double)p.K;
  }
  g.ipt = (int)((p.K + kBK - 1) / kBK);
  g.iters = (int64_t)g.num_tiles * g.ipt;
  g.issued = (double)g.iters * BM * BN * kBK;
  return g;
}

// Problem order: 1 = as given, 2 = most iterations first (stable).
std::vector<int> make_order(const std::vector<Geom>& geo, int order) {
  std::vector<int> perm(geo.size());
  std::iota(perm.begin(), perm.end(), 0);
  if (order == 2)
    std::stable_sort(perm.begin(), perm.end(),
                     [&](int a, int b) { return geo[a].iters > geo[b].iters; });
  return perm;
}

struct Config {
  int tile = 128, order = 1, grid = 0;
};

// A tuned configuration and the items it runs through the Ozaki split.
struct Tuned {
  Config cfg;
  std::vector<char> oz;
};

// Tuning results per batch signature (shapes, ops, device, options).
std::mutex g_tune_mu;
std::map<std::string, Tuned> g_tune_cache;

std::string signature(const char* device_name, const std::vector<skgemm_batch_item_t>& items,
                      const skgemm_plan_options_t& o) {
  std::string s = std::string(device_name) + "|" + std::to_string(o.tile) + "," +
                  std::to_string(o.order) + "," + std::to_string(o.grid) + "," +
                  std::to_string(o.precision) + "," + std::to_string(o.slices) + "|";
  char buf[96];
  for (const auto& it : items) {
    snprintf(buf, sizeof(buf), "%d:%lld:%lld:%lld;", it.op, (long long)it.M, (long long)it.N,
             (long long)it.K);
    s += buf;
  }
  return s;
}

}  // namespace

// ------------------------------------------------------------------ plan
struct BatchPlan {
  int device = -1;
  DeviceState* dev = nullptr;
  std::vector<skgemm_batch_item_t> items;
  std::vector<Fp64Problem> probs;
  std::vector<int> k0_items;  // items with an empty reduction and a non-empty output
  std::vector<char> oz;       // per item: runs through the Ozaki split
  // Ozaki subspace pairs: for a SYRK item the index of its GEMM partner, -2
  // for a GEMM item run by its SYRK partner, -1 otherwise.
  std::vector<int> partner;
  int slices = 0;             // Ozaki moduli (0 = accuracy target)
  int oz_precision = SKGEMM_PREC_OZAKI_I8;  // residue type of the Ozaki items
  Config cfg;
  double efficiency = 0.0;
  Fp64Group group{};
  DeviceBuffer d_probs, d_maps, d_iters, d_part, d_flags, d_err;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  int graph_kernels = 0;  // kernel nodes of the captured graph
  // Ozaki problems run on `ostream` (its scratch is the plan's), forked from
  // and joined back to the caller's stream.
  cudaStream_t ostream = nullptr;
  cudaEvent_t ofork = nullptr, ojoin = nullptr;

  int num_ozaki() const { return (int)std::count(oz.begin(), oz.end(), (char)1); }

  ~BatchPlan() {
    // Launches of the plan may still be in flight on any stream.
    cudaDeviceSynchronize();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ostream) {
      skgemm_stream_release(ostream);
      cudaStreamDestroy(ostream);
    }
    if (ofork) cudaEventDestroy(ofork);
    if (ojoin) cudaEventDestroy(ojoin);
    d_probs.release();
    d_maps.release();
    d_iters.release();
    d_part.release();
    d_flags.release();
    d_err.release();
  }
};

namespace {

int grid_cap(DeviceState* dev, int tile, int* cap) {
  int per_sm = 0;
  int st = fp64_group_occupancy(dev, tile, &per_sm);
  if (st) return st;
  *cap = dev->num_sms * per_sm;
  return SKGEMM_OK;
}

}  // namespace

// Host tables of one grouped launch: problems with work in the given order,
// their TMA descriptors for `tile` x `tile` output tiles and the iteration
// prefix.
int build_group_tables(const std::vector<Fp64Problem>& probs, int tile, int order,
                       GroupTables* T) {
  const int n = (int)probs.size();
  std::vector<Geom> geo(n);
  for (int i = 0; i < n; ++i) geo[i] = geom_of(probs[i], tile, tile);
  const std::vector<int> perm = make_order(geo, order);
  T->params.clear();
  T->maps.clear();
  T->iter_begin.assign(1, 0);
  T->params.reserve(n);
  T->maps.reserve(2 * n);
  T->useful = T->issued = 0.0;
  for (int idx : perm) {
    const Geom& g = geo[idx];
    if (g.iters == 0) continue;
    const Fp64Problem& pr = probs[idx];
    Fp64Params q;
    memset(&q, 0, sizeof(q));
    q.M = pr.M;
    q.N = pr.N;
    q.K = pr.K;
    q.tiles_m = g.tiles_m;
    q.tiles_n = g.tiles_n;
    q.num_tiles = g.num_tiles;
    q.iters_per_tile = g.ipt;
    q.total_iters = g.iters;
    q.a_kind = pr.a.kind;
    q.b_kind = pr.b.kind;
    q.tile_order = pr.tile_order;
    q.out_kind = pr.out_kind;
    q.D = pr.D;
    q.ldd = pr.ldd;
    q.alpha = pr.alpha;
    q.gamma = pr.gamma;
    q.beta_zero = pr.beta_zero ? 1 : 0;
    T->params.push_back(q);
    CUtensorMap ma, mb;
    int st;
    if ((st = make_operand_map(&ma, pr.a, pr.K, tile)) != SKGEMM_OK) return st;
    if ((st = make_operand_map(&mb, pr.b, pr.K, tile)) != SKGEMM_OK) return st;
    T->maps.push_back(ma);
    T->maps.push_back(mb);
    T->iter_begin.push_back(T->iter_begin.back() + g.iters);
    T->useful += g.useful;
    T->issued += g.issued;
  }
  if (T->iter_begin.back() > ((int64_t)1 << 40))
    return fail(SKGEMM_ERR_INVALID_ARG, "batch too large");
  return SKGEMM_OK;
}

// Cost-model tile choice: issued MACs (padding included) at a per-shape
// rate; 64 x 64 tiles carry more staging per MAC, rated 0.9 of 128 x 128.
int model_tile(const std::vector<Fp64Problem>& probs) {
  double i128 = 0.0, i64 = 0.0;
  for (const auto& pr : probs) {
    i128 += geom_of(pr, 128, 128).issued;
    i64 += geom_of(pr, 64, 64).issued;
  }
  return (i64 / 0.9 < i128) ? 64 : 128;
}

namespace {

// Pairs (SYRK i, GEMM j) with the same band-packed operand, K and M = N = M_i
// among the items flagged in `oz`: partner[i] = j, partner[j] = -2.
std::vector<int> pair_items(const std::vector<skgemm_batch_item_t>& items,
                            const std::vector<char>& oz) {
  std::vector<int> partner(items.size(), -1);
  std::map<std::tuple<const void*, int64_t, int64_t>, int> open;
  for (size_t i = 0; i < items.size(); ++i) {
    const auto& it = items[i];
    if (oz[i] && it.op == SKGEMM_OP_SYRK_PACKED && it.M > 0 && it.K > 0)
      open.emplace(std::make_tuple((const void*)it.A, it.K, it.M), (int)i);
  }
  for (size_t j = 0; j < items.size(); ++j) {
    const auto& it = items[j];
    if (!oz[j] || it.op != SKGEMM_OP_GEMM_PACKED || it.M != it.N) continue;
    auto f = open.find(std::make_tuple((const void*)it.A, it.K, it.M));
    if (f == open.end()) continue;
    partner[f->second] = (int)j;
    partner[j] = -2;
    open.erase(f);
  }
  return partner;
}

// Builds the device-side problem table, descriptors and workspace of
// configuration `c` (synchronous uploads; not during stream capture).
int configure(BatchPlan* P, Config c) {
  const int BM = c.tile, BN = c.tile;
  GroupTables T;
  std::vector<Fp64Problem> native;
  native.reserve(P->probs.size());
  for (size_t i = 0; i < P->probs.size(); ++i)
    if (!P->oz[i]) native.push_back(P->probs[i]);
  P->partner = pair_items(P->items, P->oz);
  int st0 = build_group_tables(native, c.tile, c.order, &T);
  if (st0) return st0;
  std::vector<Fp64Params>& hp = T.params;
  std::vector<CUtensorMap>& hm = T.maps;
  std::vector<int64_t>& hb = T.iter_begin;
  const double useful = T.useful, issued = T.issued;
  const int np = (int)hp.size();
  const int64_t total = hb.back();
  int cap = 0, st;
  if ((st = grid_cap(P->dev, c.tile, &cap)) != SKGEMM_OK) return st;
  int grid = c.grid > 0 ? std::min(c.grid, cap) : cap;
  grid = (int)std::min<int64_t>(grid, total);

  Fp64Group& G = P->group;
  memset(&G, 0, sizeof(G));
  G.num_problems = np;
  G.total_iters = total;
  G.grid = grid;
  if (np > 0) {
    if ((st = P->d_probs.ensure(hp.size() * sizeof(Fp64Params)))) return st;
    if ((st = P->d_maps.ensure(hm.size() * sizeof(CUtensorMap)))) return st;
    if ((st = P->d_iters.ensure(hb.size() * sizeof(int64_t)))) return st;
    if ((st = P->d_part.ensure((size_t)grid * BM * BN * sizeof(double)))) return st;
    if ((st = P->d_flags.ensure((size_t)grid * sizeof(uint32_t)))) return st;
    SKG_CUDA(cudaMemcpy(P->d_probs.ptr, hp.data(), hp.size() * sizeof(Fp64Params),
                        cudaMemcpyHostToDevice));
    SKG_CUDA(cudaMemcpy(P->d_maps.ptr, hm.data(), hm.size() * sizeof(CUtensorMap),
                        cudaMemcpyHostToDevice));
    SKG_CUDA(cudaMemcpy(P->d_iters.ptr, hb.data(), hb.size() * sizeof(int64_t),
                        cudaMemcpyHostToDevice));
  }
  if (!P->d_err.ptr) {
    if ((st = P->d_err.ensure(sizeof(uint32_t)))) return st;
    SKG_CUDA(cudaMemset(P->d_err.ptr, 0, sizeof(uint32_t)));
  }
  G.probs = (const Fp64Params*)P->d_probs.ptr;
  G.maps = (const CUtensorMap*)P->d_maps.ptr;
  G.iter_begin = (const int64_t*)P->d_iters.ptr;
  G.workspace = (double*)P->d_part.ptr;
  G.flags = (uint32_t*)P->d_flags.ptr;
  G.err = (uint32_t*)P->d_err.ptr;
  P->cfg = c;
  P->cfg.grid = grid;
  P->efficiency = issued > 0 ? useful / issued : 1.0;
  return SKGEMM_OK;
}

// One item through the Ozaki split on `s`.
int run_ozaki_item(const skgemm_batch_item_t& it, int precision, int slices, cudaStream_t s) {
  skgemm_options_t o;
  memset(&o, 0, sizeof(o));
  o.precision = precision;
  o.slices = slices;
  switch (it.op) {
    case SKGEMM_OP_GEMM_PACKED:
      return ozaki_gemm_packed(it.M, it.N, it.K, it.A, it.B, it.D, it.ldd, it.alpha, it.beta, &o,
                               s);
    case SKGEMM_OP_SYRK_PACKED:
      return ozaki_syrk_packed(it.K, it.M, it.A, it.D, it.ldd, it.alpha, it.beta, &o, s);
    case SKGEMM_OP_ROT:
      return ozaki_rot(it.M, it.N, it.A, it.B, it.D, &o, s);
    default:
      return fail(SKGEMM_ERR_INVALID_ARG, "batch item: unknown op");
  }
}

// Enqueues the plan's work on `s`: the grouped launch, the K == 0 items, then
// the Ozaki items on the plan's stream (ordered after the grouped launch).
int enqueue(BatchPlan* P, cudaStream_t s) {
  int st;
  if (P->group.num_problems > 0 &&
      (st = launch_fp64_group(P->cfg.tile, P->group, s)) != SKGEMM_OK)
    return st;
  for (int i : P->k0_items) {
    const Fp64Problem& pr = P->probs[i];
    if ((st = run_k0(pr.out_kind, pr.M, pr.N, pr.D, pr.ldd, pr.gamma, pr.beta_zero, s)))
      return st;
  }
  if (P->num_ozaki() > 0) {
    SKG_CUDA(cudaEventRecord(P->ofork, s));
    SKG_CUDA(cudaStreamWaitEvent(P->ostream, P->ofork, 0));
    for (size_t i = 0; i < P->items.size(); ++i) {
      if (!P->oz[i] || P->partner[i] == -2) continue;
      if (P->partner[i] >= 0) {
        const skgemm_batch_item_t& a = P->items[i];
        const skgemm_batch_item_t& b = P->items[P->partner[i]];
        skgemm_options_t o;
        memset(&o, 0, sizeof(o));
        o.precision = P->oz_precision;
        o.slices = P->slices;
        st = ozaki_subspace(a.K, a.M, a.A, b.B, a.D, a.ldd, a.alpha, a.beta, b.D, b.ldd, b.alpha,
                            b.beta, &o, P->ostream);
      } else {
        st = run_ozaki_item(P->items[i], P->oz_precision, P->slices, P->ostream);
      }
      if (st != SKGEMM_OK) {
        char buf[64];
        snprintf(buf, sizeof(buf), " (Ozaki item %d)", (int)i);
        const std::string msg = skgemm_last_error() + std::string(buf);
        cudaEventRecord(P->ojoin, P->ostream);
        cudaStreamWaitEvent(s, P->ojoin, 0);
        return fail(st, msg);
      }
    }
    SKG_CUDA(cudaEventRecord(P->ojoin, P->ostream));
    SKG_CUDA(cudaStreamWaitEvent(s, P->ojoin, 0));
  }
  return SKGEMM_OK;
}

int time_config(BatchPlan* P, cudaStream_t s, float* ms_out) {
  int st;
  if ((st = enqueue(P, s))) return st;  // warm-up
  cudaEvent_t e0, e1;
  SKG_CUDA(cudaEventCreate(&e0));
  SKG_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int r = 0; r < 2 && st == SKGEMM_OK; ++r) {
    cudaEventRecord(e0, s);
    st = enqueue(P, s);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "tuning run");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_out = best;
  return st;
}

int read_err(BatchPlan* P) {
  if (P->ostream) {
    // Device error word of the Ozaki kernels (kept per stream).
    int st = skgemm_stream_status(P->ostream);
    if (st) return st;
  }
  uint32_t word = 0;
  SKG_CUDA(cudaMemcpy(&word, P->d_err.ptr, sizeof(word), cudaMemcpyDeviceToHost));
  if (word == 0) return SKGEMM_OK;
  SKG_CUDA(cudaMemset(P->d_err.ptr, 0, sizeof(uint32_t)));
  char buf[160];
  snprintf(buf, sizeof(buf), "batched launch: device-side wait ran past its budget (0x%x)", word);
  return fail(SKGEMM_ERR_DEVICE_TIMEOUT, buf);
}

int build_plan(const skgemm_batch_item_t* items, int n, BatchPlan* P) {
  int st;
  P->dev = current_device(&st);
  if (!P->dev) return st;
  P->device = P->dev->device;
  if (n < 0 || (n > 0 && !items)) return fail(SKGEMM_ERR_INVALID_ARG, "bad item array");
  P->items.assign(items, items + n);
  P->probs.resize(n);
  P->oz.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    if ((st = item_problem(items[i], &P->probs[i])) != SKGEMM_OK) {
      char buf[64];
      snprintf(buf, sizeof(buf), " (item %d)", i);
      return fail(st, skgemm_last_error() + std::string(buf));
    }
    const Fp64Problem& pr = P->probs[i];
    if (pr.M > 0 && pr.N > 0 && pr.K == 0 && pr.out_kind != kOutBand16) P->k0_items.push_back(i);
  }
  return SKGEMM_OK;
}

// Cost-model time (s) of a problem's share of the grouped FP64 launch: issued
// MACs at the sustained DMMA rate (16e12 MAC/s for 128 x 128 tiles, 0.9 of it
// for 64 x 64).
double native_estimate(const Fp64Problem& p) {
  const double i128 = geom_of(p, 128, 128).issued, i64 = geom_of(p, 64, 64).issued;
  return std::min(i128 / 16e12, i64 / (0.9 * 16e12));
}

}  // namespace

double batch_native_estimate(const Fp64Problem& p) { return native_estimate(p); }

namespace {

// Items run through the Ozaki split: none (native), every one the Ozaki path
// takes (Ozaki), or those whose estimate is below 0.8 of native (auto).
std::vector<char> assign_precision(const BatchPlan& P, int precision, int slices) {
  std::vector<char> oz(P.items.size(), 0);
  if (precision == SKGEMM_PREC_NATIVE) return oz;
  for (size_t i = 0; i < P.items.size(); ++i) {
    const skgemm_batch_item_t& it = P.items[i];
    const Fp64Problem& pr = P.probs[i];
    if (pr.M == 0 || pr.N == 0 || pr.K == 0) continue;
    const int64_t n = (it.op == SKGEMM_OP_SYRK_PACKED) ? it.M : it.N;
    const double t = ozaki_time_estimate(it.op, it.M, n, it.K, slices);
    if (t < 0.0) continue;
    if (precision == SKGEMM_PREC_OZAKI_BF16) {
      if (it.op != SKGEMM_OP_ROT || it.N <= 1024) oz[i] = 1;  // BF16 rotation: nb <= 1024
      continue;
    }
    if (precision == SKGEMM_PREC_OZAKI_I8 || t < 0.8 * native_estimate(pr)) oz[i] = 1;
  }
  if (precision == SKGEMM_PREC_AUTO) {
    // Subspace pairs are priced together (one conversion of the shared operand).
    std::vector<char> all(P.items.size(), 1);
    const std::vector<int> partner = pair_items(P.items, all);
    for (size_t i = 0; i < P.items.size(); ++i) {
      const int j = partner[i];
      if (j < 0) continue;
      const skgemm_batch_item_t& it = P.items[i];
      const double t = ozaki_pair_time_estimate(it.K, it.M, slices);
      if (t < 0.0) continue;
      const char pick = t < 0.8 * (native_estimate(P.probs[i]) + native_estimate(P.probs[j]));
      oz[i] = oz[j] = pick;
    }
  }
  return oz;
}

// Copies of the SYRK outputs with beta != 0 (the product reads them), taken
// before the runs made while building a plan and written back after them.
struct SavedOutputs {
  std::vector<std::pair<int, double*>> saved;

  int save(const BatchPlan& P, cudaStream_t s) {
    for (size_t i = 0; i < P.items.size(); ++i) {
      const auto& it = P.items[i];
      if (it.op == SKGEMM_OP_SYRK_PACKED && it.beta != 0.0 && it.M > 0) {
        double* b = nullptr;
        const size_t bytes = (size_t)it.ldd * it.M * sizeof(double);
        SKG_CUDA(cudaMalloc(&b, bytes));
        saved.push_back({(int)i, b});
        SKG_CUDA(cudaMemcpyAsync(b, it.D, bytes, cudaMemcpyDeviceToDevice, s));
      }
    }
    return SKGEMM_OK;
  }
  void restore(const BatchPlan& P, cudaStream_t s) {
    for (auto& sv : saved) {
      const auto& it = P.items[sv.first];
      cudaMemcpyAsync(it.D, sv.second, (size_t)it.ldd * it.M * sizeof(double),
                      cudaMemcpyDeviceToDevice, s);
    }
    cudaStreamSynchronize(s);
    for (auto& sv : saved) cudaFree(sv.second);
    saved.clear();
  }
  ~SavedOutputs() {
    for (auto& sv : saved) cudaFree(sv.second);
  }
};

std::vector<Fp64Problem> native_subset(const BatchPlan& P) {
  std::vector<Fp64Problem> v;
  for (size_t i = 0; i < P.probs.size(); ++i)
    if (!P.oz[i]) v.push_back(P.probs[i]);
  return v;
}

}  // namespace

// Host-only schedule (exported for tests and tooling).
int batch_schedule(const skgemm_batch_item_t* items, int n, int tile, int order, int* perm_out,
                   int64_t* iter_begin_out, double* eff_out) {
  if (tile != 128 && tile != 64) return fail(SKGEMM_ERR_INVALID_ARG, "tile must be 128 or 64");
  if (order != 1 && order != 2) return fail(SKGEMM_ERR_INVALID_ARG, "order must be 1 or 2");
  if (n < 0 || (n > 0 && !items)) return fail(SKGEMM_ERR_INVALID_ARG, "bad item array");
  std::vector<Geom> geo(n);
  for (int i = 0; i < n; ++i) {
    Fp64Problem p;
    int st = item_problem(items[i], &p);
    if (st) return st;
    geo[i] = geom_of(p, tile, tile);
  }
  const std::vector<int> perm = make_order(geo, order);
  double useful = 0.0, issued = 0.0;
  int64_t acc = 0;
  for (int j = 0; j < n; ++j) {
    if (perm_out) perm_out[j] = perm[j];
    if (iter_begin_out) iter_begin_out[j] = acc;
    acc += geo[perm[j]].iters;
    useful += geo[perm[j]].useful;
    issued += geo[perm[j]].issued;
  }
  if (iter_begin_out) iter_begin_out[n] = acc;
  if (eff_out) *eff_out = issued > 0 ? useful / issued : 1.0;
  return SKGEMM_OK;
}

int plan_create(const skgemm_batch_item_t* items, int n, skgemm_plan_options_t* opts,
                cudaStream_t s, BatchPlan** out) {
  *out = nullptr;
  skgemm_plan_options_t o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  if (o.tile != 0 && o.tile != 128 && o.tile != 64)
    return fail(SKGEMM_ERR_INVALID_ARG, "plan option tile must be 0, 128 or 64");
  if (o.order < 0 || o.order > 2) return fail(SKGEMM_ERR_INVALID_ARG, "plan option order");
  if (o.grid < 0) return fail(SKGEMM_ERR_INVALID_ARG, "plan option grid");
  if (o.precision != SKGEMM_PREC_NATIVE && o.precision != SKGEMM_PREC_OZAKI_I8 &&
      o.precision != SKGEMM_PREC_AUTO && o.precision != SKGEMM_PREC_OZAKI_BF16)
    return fail(SKGEMM_ERR_INVALID_ARG, "plan option precision");
  if (o.slices != 0 && (o.slices < 6 || o.slices > 16))
    return fail(SKGEMM_ERR_INVALID_ARG, "plan option slices must be 0 or in [6, 16]");
  std::unique_ptr<BatchPlan> P(new BatchPlan());
  int st = build_plan(items, n, P.get());
  if (st) return st;
  P->use_graph = !o.no_graph;
  P->slices = o.slices;
  if (o.precision == SKGEMM_PREC_OZAKI_BF16) P->oz_precision = SKGEMM_PREC_OZAKI_BF16;

  // Precision assignments: the cost model's, and under auto also all-native
  // (tuning keeps the faster).
  std::vector<std::vector<char>> assigns;
  assigns.push_back(assign_precision(*P, o.precision, o.slices));
  const bool any_oz = std::count(assigns[0].begin(), assigns[0].end(), (char)1) > 0;
  if (o.precision == SKGEMM_PREC_AUTO && any_oz) assigns.push_back(std::vector<char>(n, 0));
  if (any_oz) {
    SKG_CUDA(cudaStreamCreateWithFlags(&P->ostream, cudaStreamNonBlocking));
    SKG_CUDA(cudaEventCreateWithFlags(&P->ofork, cudaEventDisableTiming));
    SKG_CUDA(cudaEventCreateWithFlags(&P->ojoin, cudaEventDisableTiming));
  }

  // Configuration candidates of the grouped launch.
  std::vector<Config> cands;
  for (int tile : {128, 64}) {
    if (o.tile && o.tile != tile) continue;
    for (int order : {2, 1}) {
      if (o.order && o.order != order) continue;
      Config c;
      c.tile = tile;
      c.order = order;
      c.grid = o.grid;
      cands.push_back(c);
    }
  }
  // Cost model (model_tile on the native problems): the tile with fewer
  // issued MACs per unit rate; most-work-first order.
  auto model_config = [&]() {
    Config best = cands[0];
    const int mt = model_tile(native_subset(*P));
    for (const auto& c : cands)
      if (c.tile == mt) {
        best = c;
        break;
      }
    return best;
  };
  P->oz = assigns[0];
  Tuned best{model_config(), assigns[0]};
  float best_ms = 0.f;
  int timed = 0;
  const std::string sig = signature(P->dev->name, P->items, o);
  bool cached = false;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto f = g_tune_cache.find(sig);
    // An entry (tuned here or loaded from a file) is used only if it is one
    // of the choices this plan's own tuning would time: a candidate
    // configuration and one of the precision assignments.
    bool fits = f != g_tune_cache.end() && !o.no_tune;
    if (fits) {
      bool cfg_ok = false, oz_ok = false;
      for (const auto& c : cands)
        cfg_ok |= (c.tile == f->second.cfg.tile && c.order == f->second.cfg.order &&
                   c.grid == f->second.cfg.grid);
      for (const auto& asg : assigns) oz_ok |= (asg == f->second.oz);
      fits = cfg_ok && oz_ok;
    }
    if (fits) {
      best = f->second;
      cached = true;
    }
  }
  bool has_work = false;
  for (const auto& pr : P->probs) has_work |= (pr.M > 0 && pr.N > 0);
  SavedOutputs saved;
  bool ran = false;  // the plan's work has run on `s` (scratch allocated)
  if (!o.no_tune && !cached && has_work && (cands.size() > 1 || assigns.size() > 1)) {
    if ((st = saved.save(*P, s)) != SKGEMM_OK) return st;
    float ms_best = 1e30f;
    for (const auto& asg : assigns) {
      P->oz = asg;
      bool native_work = false;
      for (const auto& pr : native_subset(*P)) native_work |= (pr.M > 0 && pr.N > 0 && pr.K > 0);
      for (size_t ci = 0; ci < cands.size() && st == SKGEMM_OK; ++ci) {
        // Without native problems the grouped configuration does not matter.
        if (!native_work && ci > 0) break;
        if ((st = configure(P.get(), cands[ci])) != SKGEMM_OK) break;
        float ms = 0.f;
        if ((st = time_config(P.get(), s, &ms)) != SKGEMM_OK) break;
        ran = true;
        ++timed;
        if (ms < ms_best) {
          ms_best = ms;
          best = Tuned{cands[ci], asg};
        }
      }
      if (st) break;
    }
    saved.restore(*P, s);
    if (st) return st;
    if ((st = read_err(P.get())) != SKGEMM_OK) return st;
    best_ms = ms_best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[sig] = best;
  }
  P->oz = best.oz;
  if ((st = configure(P.get(), best.cfg)) != SKGEMM_OK) return st;

  const bool has_oz = P->num_ozaki() > 0;
  if (P->use_graph && (P->group.num_problems > 0 || !P->k0_items.empty() || has_oz)) {
    if (has_oz && !ran) {
      // The Ozaki calls allocate their scratch, lane plans and constants on
      // first use, which stream capture does not allow: run once before.
      if ((st = saved.save(*P, s)) != SKGEMM_OK) return st;
      st = enqueue(P.get(), s);
      saved.restore(*P, s);
      if (st) return st;
      if ((st = read_err(P.get())) != SKGEMM_OK) return st;
    }
    cudaStream_t cap;
    SKG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      st = enqueue(P.get(), cap);
      cudaGraph_t g = nullptr;
      e = cudaStreamEndCapture(cap, &g);
      if (st == SKGEMM_OK && e == cudaSuccess) {
        P->graph = g;
        e = cudaGraphInstantiate(&P->exec, g, 0);
        size_t nn = 0;
        if (e == cudaSuccess) e = cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
        for (size_t i = 0; e == cudaSuccess && i < nn; ++i) {
          cudaGraphNodeType t;
          if ((e = cudaGraphNodeGetType(nodes[i], &t)) == cudaSuccess &&
              t == cudaGraphNodeTypeKernel)
            ++P->graph_kernels;
        }
      } else if (g) {
        cudaGraphDestroy(g);
      }
    }
    cudaStreamDestroy(cap);
    if (st) return st;
    if (e != cudaSuccess) return cuda_fail(e, "batch graph capture");
  }
  if (opts) {
    opts->tile_out = P->cfg.tile;
    opts->grid_out = P->cfg.grid;
    opts->order_out = P->cfg.order;
    opts->candidates_timed_out = timed;
    opts->tuned_ms_out = best_ms;
    opts->model_efficiency_out = P->efficiency;
    opts->ozaki_problems_out = P->num_ozaki();
    opts->graph_kernels_out = P->graph_kernels;
  }
  *out = P.release();
  return SKGEMM_OK;
}

int plan_run(BatchPlan* P, cudaStream_t s) {
  int cur = -1;
  SKG_CUDA(cudaGetDevice(&cur));
  if (cur != P->device) return fail(SKGEMM_ERR_INVALID_ARG, "plan belongs to another device");
  if (P->exec) {
    SKG_CUDA(cudaGraphLaunch(P->exec, s));
    return SKGEMM_OK;
  }
  return enqueue(P, s);
}

int plan_status(BatchPlan* P, cudaStream_t s) {
  SKG_CUDA(cudaStreamSynchronize(s));
  return read_err(P);
}

// One-shot grouped launch on a per-stream plan cache entry: the plan (and so
// its workspace) stays alive until the next one-shot batch on that stream has
// been ordered behind it.
namespace {
std::mutex g_oneshot_mu;
std::map<std::pair<int, cudaStream_t>, BatchPlan*> g_oneshot;
}  // namespace

int batch_dev(const skgemm_batch_item_t* items, int n, cudaStream_t s) {
  skgemm_plan_options_t o;
  memset(&o, 0, sizeof(o));
  o.no_tune = 1;
  o.no_graph = 1;
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  std::lock_guard<std::mutex> lk(g_oneshot_mu);
  BatchPlan*& slot = g_oneshot[{dev->device, s}];
  if (slot) {
    // The previous one-shot plan's launch may still be in flight on `s`:
    // its buffers are released only after the stream has passed it.
    SKG_CUDA(cudaStreamSynchronize(s));
    st = read_err(slot);
    delete slot;
    slot = nullptr;
    if (st) return st;
  }
  BatchPlan* P = nullptr;
  if ((st = plan_create(items, n, &o, s, &P)) != SKGEMM_OK) return st;
  slot = P;
  return enqueue(P, s);
}

// Device-side failures of one-shot batches on `s` (called by
// skgemm_stream_status after it has synchronised `s`).
int batch_consume_error(DeviceState* dev, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_oneshot_mu);
  auto f = g_oneshot.find({dev->device, s});
  if (f == g_oneshot.end() || !f->second) return SKGEMM_OK;
  return read_err(f->second);
}

// ---------------------------------------------------------------- ring
// A ring of grouped-launch workspaces: submission i uses slot i % depth, so a
// launch's tables and partial slots stay untouched until `depth` later
// submissions. Tables travel through pinned host memory with
// cudaMemcpyAsync on the launch stream (no host-side synchronisation unless
// the slot's previous launch is still running).
struct GroupRing {
  struct Slot {
    DeviceBuffer probs, maps, iters, part, flags, err;
    void* host = nullptr;  // pinned staging of the three tables
    size_t host_bytes = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
  };
  DeviceState* dev = nullptr;
  std::vector<Slot> slots;
  int next = 0;
};

GroupRing* group_ring_create(DeviceState* dev, int depth) {
  GroupRing* R = new GroupRing();
  R->dev = dev;
  R->slots.resize(depth < 1 ? 1 : depth);
  return R;
}

void group_ring_destroy(GroupRing* R) {
  if (!R) return;
  for (auto& sl : R->slots) {
    if (sl.ev) {
      cudaEventSynchronize(sl.ev);
      cudaEventDestroy(sl.ev);
    }
    if (sl.host) cudaFreeHost(sl.host);
    sl.probs.release();
    sl.maps.release();
    sl.iters.release();
    sl.part.release();
    sl.flags.release();
    sl.err.release();
  }
  delete R;
}

int group_ring_reserve(GroupRing* R, int max_problems) {
  if (!R) return fail(SKGEMM_ERR_INVALID_ARG, "null group ring");
  int cap128 = 0, cap64 = 0, st;
  if ((st = grid_cap(R->dev, 128, &cap128)) || (st = grid_cap(R->dev, 64, &cap64))) return st;
  const size_t part = std::max((size_t)cap128 * 128 * 128, (size_t)cap64 * 64 * 64) * 8;
  const int grid = std::max(cap128, cap64);
  for (auto& sl : R->slots) {
    if ((st = sl.probs.ensure((size_t)max_problems * sizeof(Fp64Params)))) return st;
    if ((st = sl.maps.ensure((size_t)2 * max_problems * sizeof(CUtensorMap)))) return st;
    if ((st = sl.iters.ensure((size_t)(max_problems + 1) * sizeof(int64_t)))) return st;
    if ((st = sl.part.ensure(part))) return st;
    if ((st = sl.flags.ensure((size_t)grid * sizeof(uint32_t)))) return st;
    if (!sl.err.ptr) {
      if ((st = sl.err.ensure(sizeof(uint32_t)))) return st;
      SKG_CUDA(cudaMemset(sl.err.ptr, 0, sizeof(uint32_t)));
    }
    if (!sl.ev) SKG_CUDA(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
  }
  return SKGEMM_OK;
}

int group_ring_submit(GroupRing* R, const std::vector<Fp64Problem>& probs, cudaStream_t s,
                      int* tile_out) {
  if (!R || R->slots.empty()) return fail(SKGEMM_ERR_INVALID_ARG, "null group ring");
  GroupRing::Slot& sl = R->slots[R->next];
  R->next = (R->next + 1) % (int)R->slots.size();
  if (sl.pending) {
    SKG_CUDA(cudaEventSynchronize(sl.ev));
    sl.pending = false;
  }
  const int tile = model_tile(probs);
  GroupTables T;
  int st = build_group_tables(probs, tile, 2, &T);
  if (st) return st;
  const int np = (int)T.params.size();
  if ((st = group_ring_reserve(R, np > 0 ? np : 1))) return st;
  Fp64Group g;
  memset(&g, 0, sizeof(g));
  if (np > 0) {
    const size_t bp = (size_t)np * sizeof(Fp64Params), bm = 2 * (size_t)np * sizeof(CUtensorMap),
                 bi = (size_t)(np + 1) * sizeof(int64_t);
    const size_t om = (bp + 63) / 64 * 64, oi = om + bm, need = oi + bi;
    if (sl.host_bytes < need) {
      if (sl.host) cudaFreeHost(sl.host);
      sl.host = nullptr;
      sl.host_bytes = 0;
      SKG_CUDA(cudaMallocHost(&sl.host, need));
      sl.host_bytes = need;
    }
    char* h = (char*)sl.host;
    memcpy(h, T.params.data(), bp);
    memcpy(h + om, T.maps.data(), bm);
    memcpy(h + oi, T.iter_begin.data(), bi);
    SKG_CUDA(cudaMemcpyAsync(sl.probs.ptr, h, bp, cudaMemcpyHostToDevice, s));
    SKG_CUDA(cudaMemcpyAsync(sl.maps.ptr, h + om, bm, cudaMemcpyHostToDevice, s));
    SKG_CUDA(cudaMemcpyAsync(sl.iters.ptr, h + oi, bi, cudaMemcpyHostToDevice, s));
    int cap = 0;
    if ((st = grid_cap(R->dev, tile, &cap))) return st;
    g.probs = (const Fp64Params*)sl.probs.ptr;
    g.maps = (const CUtensorMap*)sl.maps.ptr;
    g.iter_begin = (const int64_t*)sl.iters.ptr;
    g.num_problems = np;
    g.total_iters = T.iter_begin.back();
    g.grid = (int)std::min<int64_t>(cap, g.total_iters);
    g.workspace = (double*)sl.part.ptr;
    g.flags = (uint32_t*)sl.flags.ptr;
    g.err = (uint32_t*)sl.err.ptr;
    if ((st = launch_fp64_group(tile, g, s))) return st;
  }
  for (const auto& pr : probs)
    if (pr.M > 0 && pr.N > 0 && pr.K == 0 && pr.out_kind != kOutBand16)
      if ((st = run_k0(pr.out_kind, pr.M, pr.N, pr.D, pr.ldd, pr.gamma, pr.beta_zero, s)))
        return st;
  SKG_CUDA(cudaEventRecord(sl.ev, s));
  sl.pending = true;
  if (tile_out) *tile_out = tile;
  return SKGEMM_OK;
}

int group_ring_error(GroupRing* R) {
  if (!R) return SKGEMM_OK;
  for (auto& sl : R->slots) {
    if (!sl.err.ptr) continue;
    uint32_t word = 0;
    SKG_CUDA(cudaMemcpy(&word, sl.err.ptr, sizeof(word), cudaMemcpyDeviceToHost));
    if (word) {
      SKG_CUDA(cudaMemset(sl.err.ptr, 0, sizeof(uint32_t)));
      char buf[120];
      snprintf(buf, sizeof(buf), "grouped launch: device-side wait ran past its budget (0x%x)",
               word);
      return fail(SKGEMM_ERR_DEVICE_TIMEOUT, buf);
    }
  }
  return SKGEMM_OK;
}

}  // namespace skg

using namespace skg;

#define SKG_EXPORT extern "C" __attribute__((visibility("default")))

struct skgemm_plan {
  BatchPlan* impl;
};

SKG_EXPORT int skgemm_plan_create(const skgemm_batch_item_t* items, int n,
                                  skgemm_plan_options_t* opts, void* stream,
                                  skgemm_plan_t* plan_out) {
  NvtxRange nvtx_(__func__);
  if (!plan_out) return fail(SKGEMM_ERR_INVALID_ARG, "null plan_out");
  *plan_out = nullptr;
  BatchPlan* P = nullptr;
  int st = plan_create(items, n, opts, reinterpret_cast<cudaStream_t>(stream), &P);
  if (st) return st;
  *plan_out = new skgemm_plan{P};
  return SKGEMM_OK;
}

SKG_EXPORT int skgemm_plan_run(skgemm_plan_t plan, void* stream) {
  NvtxRange nvtx_(__func__);
  if (!plan || !plan->impl) return fail(SKGEMM_ERR_INVALID_ARG, "null plan");
  return plan_run(plan->impl, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_plan_status(skgemm_plan_t plan, void* stream) {
  NvtxRange nvtx_(__func__);
  if (!plan || !plan->impl) return fail(SKGEMM_ERR_INVALID_ARG, "null plan");
  return plan_status(plan->impl, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_plan_precisions(skgemm_plan_t plan, int* prec_out, int n) {
  if (!plan || !plan->impl) return fail(SKGEMM_ERR_INVALID_ARG, "null plan");
  const BatchPlan* P = plan->impl;
  if (n != (int)P->oz.size() || (n > 0 && !prec_out))
    return fail(SKGEMM_ERR_INVALID_ARG, "plan precisions: n must equal the item count");
  for (int i = 0; i < n; ++i) prec_out[i] = P->oz[i] ? P->oz_precision : SKGEMM_PREC_NATIVE;
  return SKGEMM_OK;
}

SKG_EXPORT void skgemm_plan_destroy(skgemm_plan_t plan) {
  if (!plan) return;
  delete plan->impl;
  delete plan;
}

SKG_EXPORT int skgemm_batch_dev(const skgemm_batch_item_t* items, int n, void* stream) {
  NvtxRange nvtx_(__func__);
  return batch_dev(items, n, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_batch_schedule(const skgemm_batch_item_t* items, int n, int tile,
                                     int order, int* perm_out, int64_t* iter_begin_out,
                                     double* efficiency_out) {
  return batch_schedule(items, n, tile, order, perm_out, iter_begin_out, efficiency_out);
}

// ------------------------------------------------------------ tuning cache
// The autotuner's choices (per batch signature: device name, plan options,
// each item's op and shape) as a JSON file, one entry per line:
//   {"format": "skgemm-tune-cache/1", "entries": [
//    {"key": "<signature>", "tile": 128, "order": 1, "grid": 0, "ozaki": "0101"},
//    ...]}
// so that a serving process or a solver restarted on the same device type
// skips the timing runs of plans it has tuned before.
namespace {
const char* kTuneFormat = "skgemm-tune-cache/1";

// The text after `"name": ` on `line` (its quoted string, or its integer).
bool json_string(const std::string& line, const char* name, std::string* out) {
  const std::string tag = std::string("\"") + name + "\": \"";
  const size_t a = line.find(tag);
  if (a == std::string::npos) return false;
  const size_t b = line.find('"', a + tag.size());
  if (b == std::string::npos) return false;
  *out = line.substr(a + tag.size(), b - a - tag.size());
  return true;
}
bool json_int(const std::string& line, const char* name, int* out) {
  const std::string tag = std::string("\"") + name + "\": ";
  const size_t a = line.find(tag);
  if (a == std::string::npos) return false;
  char* end = nullptr;
  const long v = strtol(line.c_str() + a + tag.size(), &end, 10);
  if (end == line.c_str() + a + tag.size()) return false;
  *out = (int)v;
  return true;
}
}  // namespace

SKG_EXPORT int skgemm_tune_cache_save(const char* path) {
  if (!path) return fail(SKGEMM_ERR_INVALID_ARG, "tune cache: null path");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  FILE* f = fopen(path, "w");
  if (!f) return fail(SKGEMM_ERR_INVALID_ARG, std::string("tune cache: cannot write ") + path);
  fprintf(f, "{\"format\": \"%s\", \"entries\": [\n", kTuneFormat);
  size_t i = 0;
  for (const auto& kv : g_tune_cache) {
    std::string oz(kv.second.oz.size(), '0');
    for (size_t j = 0; j < oz.size(); ++j) oz[j] = kv.second.oz[j] ? '1' : '0';
    fprintf(f, "{\"key\": \"%s\", \"tile\": %d, \"order\": %d, \"grid\": %d, \"ozaki\": \"%s\"}%s\n",
            kv.first.c_str(), kv.second.cfg.tile, kv.second.cfg.order, kv.second.cfg.grid,
            oz.c_str(), ++i < g_tune_cache.size() ? "," : "");
  }
  fprintf(f, "]}\n");
  const bool ok = fclose(f) == 0;
  if (!ok) return fail(SKGEMM_ERR_INVALID_ARG, std::string("tune cache: write failed: ") + path);
  return (int)g_tune_cache.size();
}

SKG_EXPORT int skgemm_tune_cache_load(const char* path) {
  if (!path) return fail(SKGEMM_ERR_INVALID_ARG, "tune cache: null path");
  FILE* f = fopen(path, "r");
  if (!f) return fail(SKGEMM_ERR_INVALID_ARG, std::string("tune cache: cannot read ") + path);
  std::vector<std::pair<std::string, Tuned>> got;
  std::string line;
  bool header = false, bad = false;
  char buf[4096];
  while (fgets(buf, sizeof(buf), f)) {
    // One entry per line, of any length (a batch of many items has a long key).
    line.assign(buf);
    while (!line.empty() && line.back() != '\n' && fgets(buf, sizeof(buf), f)) line += buf;
    if (!header) {
      std::string fmt;
      header = json_string(line, "format", &fmt) && fmt == kTuneFormat;
      if (!header) {
        bad = true;
        break;
      }
      continue;
    }
    if (line.find("\"key\"") == std::string::npos) continue;
    std::string key, oz;
    Tuned t;
    if (!json_string(line, "key", &key) || !json_int(line, "tile", &t.cfg.tile) ||
        !json_int(line, "order", &t.cfg.order) || !json_int(line, "grid", &t.cfg.grid) ||
        !json_string(line, "ozaki", &oz) || (t.cfg.tile != 64 && t.cfg.tile != 128) ||
        t.cfg.grid < 0 || t.cfg.order < 0) {
      bad = true;
      break;
    }
    for (char c : oz) {
      if (c != '0' && c != '1') bad = true;
      t.oz.push_back(c == '1' ? 1 : 0);
    }
    if (bad) break;
    got.emplace_back(key, t);
  }
  fclose(f);
  if (bad || !header)
    return fail(SKGEMM_ERR_INVALID_ARG, std::string("tune cache: not a skgemm tuning file: ") + path);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto& e : got) g_tune_cache[e.first] = e.second;
  return (int)got.size();
}

SKG_EXPORT int skgemm_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache.clear();
  return SKGEMM_OK;
}
