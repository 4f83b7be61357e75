// Grouped mixed-length C2C plans: task lists for grouped.cu, FP64 tables,
// CUDA-graph replay, and the plfft_cuda_group_* C-ABI.
//
// Per transform of length n the schedule is (the same strategy order as the
// single-length planner, src/planner/planner.cpp:49-182):
//   smooth n on chip                      -> one GT_TILE task        (phase 0)
//   prime n, smooth n-1 on chip           -> one GT_RADER task       (phase 0)
//   Bluestein length M = smooth >= 2n-1 on chip -> one GT_BLUE task  (phase 0)
//   smooth n too long for one CTA         -> four-step column tiles (phase 0)
//                                            and row tiles (phase 1)
//   Rader / Bluestein with a convolution too long for one CTA
//                                         -> forward four-step tiles with the
//                                            gather/chirp prologue (phase 0),
//                                            row tiles with the spectrum
//                                            product (1), inverse column tiles
//                                            (2), inverse row tiles with the
//                                            scatter/chirp epilogue (3).
// Phases are consecutive launches of the persistent kernel, captured once in a
// CUDA graph per (input, output) pointer pair and replayed.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>

#include "../../include/plfft.h"
#include "../../include/plfft_cuda.h"
#include "plan.hpp"

namespace plfft_b200 {

namespace {

constexpr int kGroupOnChip = 8192;  // longest on-chip length of the grouped kernel
constexpr int kGroupE = 32;
constexpr int kGroupThr = 256;
constexpr int kPhases = 4;

bool tile_fits(int L, int cnt, const std::vector<int>& radices) {
  for (int R : radices)
    if (int64_t(cnt) * (L / R) > int64_t(kGroupE / R) * kGroupThr) return false;
  return int64_t(cnt) * spad_len(L) <= group_max_smem_elems();
}

struct Tables {
  DevBuf perm_in, perm_out, spec, chirp;
};

}  // namespace

// Schedule of a grouped execution (the autotuner's choices): columns or rows
// per four-step tile, same-length on-chip transforms merged into one task,
// largest radix of the on-chip stage lists.
struct GroupShape {
  // measured on the 4000-transform mix: 32-wide tiles 1.15x over 16, 8 at
  // 0.77x; merging 1.02x; radix 8 or 32 below 16
  int tile_cap = 32;
  int merge_cap = 16;
  int max_radix = 16;
  std::string str() const {
    std::ostringstream o;
    o << "tile=" << tile_cap << " merge=" << merge_cap << " radix=" << max_radix;
    return o.str();
  }
};

struct GroupData {
  int device = 0;
  int dir = -1;
  GroupShape shape;
  int64_t count = 0;
  std::vector<GTask> tasks[kPhases];
  DevBuf tasks_dev[kPhases];
  std::vector<FftDesc> descs;
  std::vector<std::unique_ptr<DevBuf>> tws;
  std::map<int, int> desc_of;
  DevBuf descs_dev, tws_dev;
  std::map<int64_t, std::unique_ptr<Tables>> rader, blue;
  std::map<int64_t, std::unique_ptr<DevBuf>> lo, hi;  // two-level tables per length
  std::map<int64_t, int> lbits;
  DevBuf counters;
  DevBuf ws;
  size_t ws_bytes = 0;
  int smem_bytes = 0;
  int grid[kPhases] = {0, 0, 0, 0};
  int nlarge = 0, nonchip = 0, nrader = 0, nblue = 0, nconv_large = 0;
  bool use_graph = true;
  cudaGraphExec_t graph = nullptr;
  const void* graph_in = nullptr;
  void* graph_out = nullptr;
  std::string why;

  ~GroupData() {
    if (graph) cudaGraphExecDestroy(graph);
  }

  int desc(int L) {
    auto it = desc_of.find(L);
    if (it != desc_of.end()) return it->second;
    std::vector<float2> tw;
    const FftDesc d = make_desc(L, factor_radices(L, shape.max_radix), tw);
    auto buf = std::make_unique<DevBuf>();
    if (buf->upload(tw) != cudaSuccess) return -1;
    descs.push_back(d);
    tws.push_back(std::move(buf));
    const int idx = int(descs.size()) - 1;
    desc_of[L] = idx;
    return idx;
  }

  bool onchip(int64_t L, int cnt = 1) {
    if (L > kGroupOnChip || !is_smooth(L)) return false;
    return tile_fits(int(L), cnt, factor_radices(L, shape.max_radix));
  }

  // largest tile count that fits for length L (up to cap)
  int tile_count(int L, int cap) {
    int c = cap;
    while (c > 1 && !tile_fits(L, c, factor_radices(L, shape.max_radix))) --c;
    return c;
  }

  TwoLevel two_level(int64_t n) {
    auto it = lo.find(n);
    if (it == lo.end()) {
      int64_t L = int64_t(1);
      int b = 0;
      while ((int64_t(1) << b) < n) ++b;
      L = int64_t(1) << ((b + 1) / 2);
      std::vector<float2> l(L), h((n + L - 1) / L);
      for (int64_t i = 0; i < L; ++i) {
        double c, s;
        unit_root(i, n, c, s);
        l[i] = make_float2(float(c), float(-s));
      }
      for (size_t i = 0; i < h.size(); ++i) {
        double c, s;
        unit_root(int64_t(i) * L, n, c, s);
        h[i] = make_float2(float(c), float(-s));
      }
      auto a = std::make_unique<DevBuf>();
      auto bb = std::make_unique<DevBuf>();
      a->upload(l);
      bb->upload(h);
      lo[n] = std::move(a);
      hi[n] = std::move(bb);
      lbits[n] = int(L);
    }
    return TwoLevel{lo[n]->as<float2>(), hi[n]->as<float2>(), n, lbits[n]};
  }

  Tables* rader_tables(int64_t p) {
    auto& t = rader[p];
    if (t) return t.get();
    t = std::make_unique<Tables>();
    const int64_t m = p - 1;
    const int64_t g = primitive_root(p), ginv = pow_mod(g, p - 2, p);
    std::vector<int> pin(m), pout(m);
    std::vector<cd> b(m);
    int64_t gq = 1, gi = 1;
    for (int64_t q = 0; q < m; ++q) {
      pin[q] = int(gq);
      pout[q] = int(gi);
      double c, s;
      unit_root(gi, p, c, s);
      b[q] = cd(c, dir * s);
      gq = gq * g % p;
      gi = gi * ginv % p;
    }
    t->perm_in.upload(pin);
    t->perm_out.upload(pout);
    t->spec.upload(to_f2(host_fft(b, -1), 1.0 / double(m)));
    return t.get();
  }

  Tables* blue_tables(int64_t n, int64_t m) {
    auto& t = blue[n];
    if (t) return t.get();
    t = std::make_unique<Tables>();
    std::vector<cd> w(n), b(m, cd(0, 0));
    for (int64_t k = 0; k < n; ++k) {
      const int64_t e = int64_t((__int128)k * k % (2 * n));
      double c, s;
      unit_root(e, 2 * n, c, s);
      w[k] = cd(c, dir * s);
    }
    for (int64_t k = 0; k < n; ++k) {
      b[k] = std::conj(w[k]);
      if (k) b[m - k] = std::conj(w[k]);
    }
    t->chirp.upload(to_f2(w, 1.0));
    t->spec.upload(to_f2(host_fft(b, -1), 1.0 / double(m)));
    return t.get();
  }

  // split m = m1 * m2 for tiles: m1 (column length) small for coalesced
  // column tiles, both on chip
  bool split(int64_t m, int64_t& m1, int64_t& m2) {
    int64_t best = 0;
    for (int64_t d = 2; d * d <= m; ++d) {
      if (m % d) continue;
      if (onchip(d, 1) && onchip(m / d, 1)) best = d;
    }
    if (!best) return false;
    m1 = best;
    m2 = m / best;
    return true;
  }

  GTask base_task(int type, int dir_, int n, int cnt, int d) {
    GTask T;
    std::memset(&T, 0, sizeof(T));
    T.type = type;
    T.dir = dir_;
    T.n = n;
    T.cnt = cnt;
    T.desc = d;
    T.scale = 1.f;
    T.tw2 = TwoLevel{nullptr, nullptr, 1, 1};
    return T;
  }

  // four-step tiles of a length-m transform: columns from (in_buf, in_off)
  // into scratch s1, rows from s1 into (out_buf, out_off).  Returns false if
  // m cannot be split.
  bool add_four_step(int64_t m, int tdir, int pcol, int prow, int in_buf, int64_t in_off, int out_buf, int64_t out_off,
                     int64_t s1, const GTask& pro, const GTask& epi) {
    int64_t m1, m2;
    if (!split(m, m1, m2)) return false;
    const int d1 = desc(int(m1)), d2 = desc(int(m2));
    if (d1 < 0 || d2 < 0) return false;
    const TwoLevel tl = two_level(m);
    const int c1 = tile_count(int(m1), shape.tile_cap), c2 = tile_count(int(m2), shape.tile_cap);
    for (int64_t col0 = 0; col0 < m2; col0 += c1) {
      GTask T = base_task(GT_TILE, tdir, int(m1), int(std::min<int64_t>(c1, m2 - col0)), d1);
      T.in_buf = in_buf;
      T.in_off = in_off + (pro.pre_op == GO_GATHER ? 0 : col0);
      T.icdist = 1;
      T.ikstride = pro.pre_op == GO_GATHER ? 1 : m2;
      T.pre_op = pro.pre_op;
      T.pre_len = pro.pre_len;
      T.pre_tab = pro.pre_tab;
      T.perm_in = pro.perm_in;
      T.ie0 = col0;
      T.iec = 1;
      T.iek = m2;
      T.out_buf = 2;
      T.out_off = s1 + col0;
      T.ocdist = 1;
      T.okstride = m2;
      T.post_op = GO_TWIDDLE;
      T.col0 = col0;
      T.tw2 = tl;
      tasks[pcol].push_back(T);
    }
    for (int64_t row0 = 0; row0 < m1; row0 += c2) {
      GTask T = base_task(GT_TILE, tdir, int(m2), int(std::min<int64_t>(c2, m1 - row0)), d2);
      T.in_buf = 2;
      T.in_off = s1 + row0 * m2;
      T.icdist = m2;
      T.ikstride = 1;
      T.out_buf = out_buf;
      const bool natural = epi.post_op != GO_SCATTER;
      T.out_off = out_off + (natural ? row0 : 0);
      T.ocdist = 1;
      T.okstride = natural ? m1 : 1;
      T.oe0 = row0;
      T.oec = 1;
      T.oek = m1;
      T.post_op = epi.post_op;
      T.post_tab = epi.post_tab;
      T.post_len = epi.post_len;
      T.perm_out = epi.perm_out;
      T.sum0 = epi.sum0;
      T.aux_buf = epi.aux_buf;
      T.aux_off = epi.aux_off;
      if (epi.post_op == GO_SCATTER) {
        T.ocdist = 0;  // scatter addresses come from perm_out
      }
      tasks[prow].push_back(T);
    }
    return true;
  }

  bool build(int64_t cnt, const int64_t* lengths, const int64_t* in_offs, const int64_t* out_offs) {
    count = cnt;
    // scratch layout for the long transforms
    std::vector<int64_t> s_off(cnt, -1);
    size_t ws_elems = 0;
    auto reserve = [&](int64_t elems) {
      const int64_t off = int64_t(ws_elems);
      ws_elems += size_t((elems + 31) & ~int64_t(31));
      return off;
    };
    struct Plan {
      int kind;  // 0 onchip, 1 rader, 2 blue, 3 four-step, 4 big rader, 5 big blue
      int64_t m;
    };
    std::vector<Plan> plans(cnt);
    for (int64_t i = 0; i < cnt; ++i) {
      const int64_t n = lengths[i];
      if (n < 1) {
        why = "length must be positive";
        return false;
      }
      if (onchip(n)) {
        plans[i] = {0, n};
      } else if (is_smooth(n)) {
        plans[i] = {3, n};
      } else if (is_prime(n) && n > 2 && is_smooth(n - 1)) {
        plans[i] = {onchip(n - 1) ? 1 : 4, n - 1};
      } else {
        const int64_t m = next_smooth(2 * n - 1);
        plans[i] = {onchip(m) ? 2 : 5, m};
      }
    }
    // one slot per transform for the long ones (sum0 slots at the end)
    std::vector<int64_t> sum_off(cnt, -1);
    for (int64_t i = 0; i < cnt; ++i) {
      if (plans[i].kind == 3) s_off[i] = reserve(plans[i].m);
      if (plans[i].kind >= 4) s_off[i] = reserve(2 * plans[i].m);
      if (plans[i].kind == 4) sum_off[i] = reserve(1);
    }
    ws_bytes = std::max<size_t>(ws_elems * sizeof(float2), 256);
    if (ws.alloc(ws_bytes) != cudaSuccess) {
      why = "workspace allocation failed";
      return false;
    }
    float2* wsp = ws.as<float2>();
    for (int64_t i = 0; i < cnt; ++i) {
      const int64_t n = lengths[i];
      const Plan& pl = plans[i];
      if (pl.kind == 0) {
        // transforms i, i+1, ... of the same length whose offsets step by
        // the same distances (>= n, so members do not overlap) share a task
        int run = 1;
        if (shape.merge_cap > 1) {
          const int cap = tile_count(int(n), shape.merge_cap);
          const int64_t di = i + 1 < cnt ? in_offs[i + 1] - in_offs[i] : 0;
          const int64_t dout = i + 1 < cnt ? out_offs[i + 1] - out_offs[i] : 0;
          while (run < cap && i + run < cnt && plans[i + run].kind == 0 && lengths[i + run] == n &&
                 in_offs[i + run] - in_offs[i + run - 1] == di && out_offs[i + run] - out_offs[i + run - 1] == dout &&
                 di >= n && dout >= n)
            ++run;
        }
        GTask T = base_task(GT_TILE, dir, int(n), run, desc(int(n)));
        T.in_buf = 0;
        T.in_off = in_offs[i];
        T.ikstride = 1;
        T.icdist = run > 1 ? in_offs[i + 1] - in_offs[i] : n;
        T.out_buf = 1;
        T.out_off = out_offs[i];
        T.okstride = 1;
        T.ocdist = run > 1 ? out_offs[i + 1] - out_offs[i] : n;
        tasks[0].push_back(T);
        nonchip += run;
        i += run - 1;
      } else if (pl.kind == 1) {
        Tables* t = rader_tables(n);
        GTask T = base_task(GT_RADER, dir, int(pl.m), 1, desc(int(pl.m)));
        T.in_buf = 0;
        T.in_off = in_offs[i];
        T.ikstride = 1;
        T.out_buf = 1;
        T.out_off = out_offs[i];
        T.okstride = 1;
        T.perm_in = t->perm_in.as<int>();
        T.perm_out = t->perm_out.as<int>();
        T.post_tab = t->spec.as<float2>();
        tasks[0].push_back(T);
        ++nrader;
      } else if (pl.kind == 2) {
        Tables* t = blue_tables(n, pl.m);
        GTask T = base_task(GT_BLUE, dir, int(pl.m), 1, desc(int(pl.m)));
        T.in_buf = 0;
        T.in_off = in_offs[i];
        T.ikstride = 1;
        T.out_buf = 1;
        T.out_off = out_offs[i];
        T.okstride = 1;
        T.pre_len = int(n);
        T.pre_tab = t->chirp.as<float2>();
        T.post_tab2 = t->spec.as<float2>();
        tasks[0].push_back(T);
        ++nblue;
      } else if (pl.kind == 3) {
        GTask none = base_task(GT_TILE, dir, 0, 0, 0);
        if (!add_four_step(n, dir, 0, 1, 0, in_offs[i], 1, out_offs[i], s_off[i], none, none)) {
          why = "length " + std::to_string(n) + " has no grouped schedule";
          return false;
        }
        ++nlarge;
      } else {
        // long convolution: forward FFT_M (phases 0, 1), inverse (2, 3)
        const int64_t m = pl.m;
        const int64_t s1 = s_off[i], s2 = s_off[i] + m;
        GTask pro = base_task(GT_TILE, -1, 0, 0, 0), epi1 = pro, pro2 = pro, epi2 = pro;
        if (pl.kind == 4) {
          Tables* t = rader_tables(n);
          pro.pre_op = GO_GATHER;
          pro.perm_in = t->perm_in.as<int>();
          epi1.post_op = GO_SPEC_SAVE0;
          epi1.post_tab = t->spec.as<float2>();
          epi1.sum0 = wsp + sum_off[i];
          epi2.post_op = GO_SCATTER;
          epi2.perm_out = t->perm_out.as<int>();
          epi2.sum0 = wsp + sum_off[i];
          epi2.aux_buf = 0;
          epi2.aux_off = in_offs[i];
        } else {
          Tables* t = blue_tables(n, m);
          pro.pre_op = GO_CHIRP;
          pro.pre_tab = t->chirp.as<float2>();
          pro.pre_len = int(n);
          epi1.post_op = GO_SPEC;
          epi1.post_tab = t->spec.as<float2>();
          epi2.post_op = GO_CHIRP;
          epi2.post_tab = t->chirp.as<float2>();
          epi2.post_len = int(n);
        }
        const bool ok = add_four_step(m, -1, 0, 1, 0, in_offs[i], 2, s2, s1, pro, epi1) &&
                        add_four_step(m, +1, 2, 3, 2, s2, 1, out_offs[i], s1, pro2, epi2);
        if (!ok) {
          why = "convolution length " + std::to_string(m) + " has no grouped schedule";
          return false;
        }
        ++nconv_large;
      }
    }
    // device copies of descriptors, twiddle pointers, tasks (longest first)
    std::vector<const float2*> twp(tws.size());
    for (size_t k = 0; k < tws.size(); ++k) twp[k] = tws[k]->as<float2>();
    if (descs_dev.upload(descs) != cudaSuccess || tws_dev.upload(twp) != cudaSuccess) return false;
    int max_elems = 1;
    for (int p = 0; p < kPhases; ++p) {
      auto cost = [](const GTask& t) {
        double c = double(t.cnt) * t.n * std::log2(double(t.n) + 1.0);
        return t.type == GT_TILE ? c : 2.0 * c;
      };
      std::stable_sort(tasks[p].begin(), tasks[p].end(),
                       [&](const GTask& a, const GTask& b) { return cost(a) > cost(b); });
      for (const GTask& t : tasks[p]) max_elems = std::max(max_elems, t.cnt * spad_len(t.n));
      if (!tasks[p].empty() && tasks_dev[p].upload(tasks[p]) != cudaSuccess) return false;
    }
    smem_bytes = max_elems * int(sizeof(float2));
    if (counters.alloc(2 * kPhases * sizeof(int)) != cudaSuccess ||
        cudaMemset(counters.p, 0, 2 * kPhases * sizeof(int)) != cudaSuccess)
      return false;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int per = grouped_blocks_per_sm(smem_bytes);
    for (int p = 0; p < kPhases; ++p)
      grid[p] = int(std::min<int64_t>(int64_t(tasks[p].size()), int64_t(per) * sms));
    return true;
  }

  cudaError_t launch_all(const void* in, void* out, cudaStream_t st) {
    for (int p = 0; p < kPhases; ++p) {
      if (tasks[p].empty()) continue;
      GroupPhase P{};
      P.tasks = tasks_dev[p].as<GTask>();
      P.ntasks = int(tasks[p].size());
      P.descs = descs_dev.as<FftDesc>();
      P.tws = tws_dev.as<const float2*>();
      P.bases[0] = const_cast<float2*>(static_cast<const float2*>(in));
      P.bases[1] = static_cast<float2*>(out);
      P.bases[2] = ws.as<float2>();
      P.counter = counters.as<int>() + 2 * p;
      P.done = counters.as<int>() + 2 * p + 1;
      const cudaError_t e = launch_grouped(P, grid[p], smem_bytes, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  int launches() const {
    int n = 0;
    for (int p = 0; p < kPhases; ++p) n += tasks[p].empty() ? 0 : 1;
    return n;
  }

  cudaError_t execute(const void* in, void* out, cudaStream_t st) {
    if (!use_graph) return launch_all(in, out, st);
    if (!graph || graph_in != in || graph_out != out) {
      if (graph) {
        cudaGraphExecDestroy(graph);
        graph = nullptr;
      }
      cudaStream_t cap = nullptr;
      cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
      if (e != cudaSuccess) return e;
      cudaGraph_t g = nullptr;
      e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const cudaError_t le = launch_all(in, out, cap);
        e = cudaStreamEndCapture(cap, &g);
        if (le != cudaSuccess) e = le;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&graph, g, 0);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(cap);
      if (e != cudaSuccess) return e;
      graph_in = in;
      graph_out = out;
    }
    return cudaGraphLaunch(graph, st);
  }

  std::string describe() const {
    std::ostringstream o;
    o << "(group count=" << count << " " << shape.str() << " onchip=" << nonchip << " rader=" << nrader << " bluestein=" << nblue
      << " four-step=" << nlarge << " long-conv=" << nconv_large << " phases=" << launches() << " tasks=["
      << tasks[0].size() << "," << tasks[1].size() << "," << tasks[2].size() << "," << tasks[3].size()
      << "] smem=" << smem_bytes << " graph=" << (use_graph ? 1 : 0) << ")";
    return o.str();
  }
};

}  // namespace plfft_b200

using namespace plfft_b200;

struct plfft_cuda_group_t {
  GroupData g;
};

extern "C" {

plfft_status_t plfft_cuda_group_create(plfft_cuda_group_t** group, int64_t count, const int64_t* lengths,
                                       const int64_t* in_offsets, const int64_t* out_offsets,
                                       plfft_direction_t direction) {
  if (!group) return PLFFT_NULL_ARGUMENT;
  *group = nullptr;
  if (!lengths || !in_offsets || !out_offsets) return PLFFT_NULL_ARGUMENT;
  if (count < 1) return PLFFT_UNSUPPORTED_BATCH;
  if (direction != PLFFT_FORWARD && direction != PLFFT_BACKWARD) return PLFFT_INVALID_TRANSFORM_KIND;
  for (int64_t i = 0; i < count; ++i)
    if (lengths[i] < 1) return PLFFT_INVALID_SIZE;
  auto* h = new plfft_cuda_group_t;
  cudaGetDevice(&h->g.device);
  h->g.dir = int(direction);
  h->g.use_graph = std::getenv("PLFFT_B200_GROUP_NOGRAPH") == nullptr;
  // PLFFT_B200_GROUP_SHAPE=tile,merge,radix: a schedule other than the default
  if (const char* v = std::getenv("PLFFT_B200_GROUP_SHAPE")) {
    int a = 0, b = 0, c = 0;
    if (std::sscanf(v, "%d,%d,%d", &a, &b, &c) == 3 && a >= 1 && b >= 1 && (c == 8 || c == 16 || c == 32)) {
      h->g.shape.tile_cap = a;
      h->g.shape.merge_cap = b;
      h->g.shape.max_radix = c;
    }
  }
  if (!h->g.build(count, lengths, in_offsets, out_offsets)) {
    delete h;
    return PLFFT_PLAN_CREATION_FAILED;
  }
  *group = h;
  return PLFFT_OK;
}

plfft_status_t plfft_cuda_group_execute_async(plfft_cuda_group_t* group, const void* d_input, void* d_output,
                                              void* stream) {
  if (!group || !d_input || !d_output) return PLFFT_NULL_ARGUMENT;
  const cudaError_t e = group->g.execute(d_input, d_output, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? PLFFT_OK : PLFFT_CUDA_ERROR;
}

plfft_status_t plfft_cuda_group_create_tuned(plfft_cuda_group_t** group, int64_t count, const int64_t* lengths,
                                             const int64_t* in_offsets, const int64_t* out_offsets,
                                             plfft_direction_t direction, plfft_rigor_t rigor) {
  if (rigor == PLFFT_ESTIMATE) return plfft_cuda_group_create(group, count, lengths, in_offsets, out_offsets, direction);
  if (!group) return PLFFT_NULL_ARGUMENT;
  *group = nullptr;
  if (!lengths || !in_offsets || !out_offsets) return PLFFT_NULL_ARGUMENT;
  if (count < 1) return PLFFT_UNSUPPORTED_BATCH;
  if (direction != PLFFT_FORWARD && direction != PLFFT_BACKWARD) return PLFFT_INVALID_TRANSFORM_KIND;
  if (rigor != PLFFT_MEASURE && rigor != PLFFT_PATIENT && rigor != PLFFT_EXHAUSTIVE) return PLFFT_INVALID_PLANNER_RIGOR;
  for (int64_t i = 0; i < count; ++i)
    if (lengths[i] < 1) return PLFFT_INVALID_SIZE;
  int device = 0;
  cudaGetDevice(&device);
  const bool use_graph = std::getenv("PLFFT_B200_GROUP_NOGRAPH") == nullptr;
  auto make = [&](const GroupShape& sh) -> plfft_cuda_group_t* {
    auto* h = new plfft_cuda_group_t;
    h->g.device = device;
    h->g.dir = int(direction);
    h->g.use_graph = use_graph;
    h->g.shape = sh;
    if (!h->g.build(count, lengths, in_offsets, out_offsets)) {
      delete h;
      return nullptr;
    }
    return h;
  };
  // candidate schedules, the default first: more at each rigor level
  std::vector<GroupShape> cands;
  auto add = [&](int tile, int merge, int radix) {
    GroupShape sh;
    sh.tile_cap = tile;
    sh.merge_cap = merge;
    sh.max_radix = radix;
    cands.push_back(sh);
  };
  add(32, 16, 16);
  add(16, 16, 16);
  add(64, 16, 16);
  add(32, 1, 16);
  if (rigor >= PLFFT_PATIENT) {
    add(32, 16, 8);
    add(32, 16, 32);
  }
  if (rigor >= PLFFT_EXHAUSTIVE) {
    add(8, 16, 16);
    add(16, 1, 16);
    add(32, 64, 16);
    add(64, 64, 16);
  }
  // the problem's key: FNV-1a over lengths and offsets, the count, direction, device
  uint64_t hsh = 1469598103934665603ull;
  auto mix = [&](int64_t v) {
    for (int b = 0; b < 8; ++b) {
      hsh ^= uint64_t(v >> (8 * b)) & 0xffu;
      hsh *= 1099511628211ull;
    }
  };
  int64_t in_span = 0, out_span = 0;
  for (int64_t i = 0; i < count; ++i) {
    mix(lengths[i]);
    mix(in_offsets[i]);
    mix(out_offsets[i]);
    in_span = std::max(in_span, in_offsets[i] + lengths[i]);
    out_span = std::max(out_span, out_offsets[i] + lengths[i]);
  }
  std::ostringstream key;
  key << "group count=" << count << " hash=" << std::hex << hsh << std::dec << " dir=" << int(direction)
      << " dev=" << wisdom_device();
  std::string known;
  if (wisdom_recall(key.str(), known))
    for (const GroupShape& sh : cands)
      if (sh.str() == known) {
        if (auto* h = make(sh)) {
          *group = h;
          return PLFFT_OK;
        }
      }
  // time each candidate on scratch buffers with the group's spans: one
  // warm-up, then executions until its share of the budget is spent (3 at
  // least); a challenger replaces the incumbent only if >= 2% faster
  const double budget = rigor == PLFFT_MEASURE ? 0.1 : (rigor == PLFFT_PATIENT ? 0.5 : 2.0);
  DevBuf din, dout;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool scratch = din.alloc(size_t(in_span) * sizeof(float2)) == cudaSuccess &&
                       dout.alloc(size_t(out_span) * sizeof(float2)) == cudaSuccess &&
                       cudaMemset(din.p, 0, size_t(in_span) * sizeof(float2)) == cudaSuccess &&
                       cudaStreamCreate(&st) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
                       cudaEventCreate(&e1) == cudaSuccess;
  plfft_cuda_group_t* best = nullptr;
  double best_t = -1;
  if (scratch) {
    const double share = budget / double(cands.size());
    for (const GroupShape& sh : cands) {
      plfft_cuda_group_t* h = make(sh);
      if (!h) continue;
      double t = -1;
      if (h->g.launch_all(din.p, dout.p, st) == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess) {
        double spent = 0;
        int reps = 0;
        while (reps < 3 || (spent < share && reps < 64)) {
          cudaEventRecord(e0, st);
          if (h->g.launch_all(din.p, dout.p, st) != cudaSuccess) break;
          cudaEventRecord(e1, st);
          if (cudaEventSynchronize(e1) != cudaSuccess) break;
          float ms = 0;
          cudaEventElapsedTime(&ms, e0, e1);
          const double sec = ms * 1e-3;
          t = t < 0 ? sec : std::min(t, sec);
          spent += sec;
          ++reps;
        }
      }
      cudaGetLastError();
      if (t > 0 && (best_t < 0 || t < best_t * 0.98)) {
        delete best;
        best = h;
        best_t = t;
      } else {
        delete h;
      }
    }
  } else {
    cudaGetLastError();
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  if (!best) best = make(cands[0]);  // no room or time to measure: the default schedule
  if (!best) return PLFFT_PLAN_CREATION_FAILED;
  if (best_t > 0) wisdom_remember(key.str(), best->g.shape.str());
  *group = best;
  return PLFFT_OK;
}

int plfft_cuda_group_get_launch_count(const plfft_cuda_group_t* group) { return group ? group->g.launches() : 0; }

plfft_status_t plfft_cuda_group_describe(const plfft_cuda_group_t* group, char* buf, size_t len) {
  if (!group || !buf) return PLFFT_NULL_ARGUMENT;
  if (len == 0) return PLFFT_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", group->g.describe().c_str());
  return PLFFT_OK;
}

void plfft_cuda_group_destroy(plfft_cuda_group_t* group) { delete group; }

}  // extern "C"
