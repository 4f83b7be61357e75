// Plan construction per (kind, data type) and synchronous execution.
//
// Dispatch mirrors reference src/plfft.cpp:488-513 (dtype x kind) and
// src/arm_fft1d_impl.hpp:109-147 (R2R wrapper, n == 1 copy); buffer spans
// follow docs/plfft.md:100-166.
#include "plan_kinds.hpp"

#include <cstring>

namespace plfft_b200 {

static int scalar_bytes(plfft_data_type_t t) {
  switch (t) {
    case PLFFT_DATA_TYPE_FP32: return 4;
    case PLFFT_DATA_TYPE_FP64: return 8;
    case PLFFT_DATA_TYPE_FP16: return 2;
    case PLFFT_DATA_TYPE_Q7: return 1;
    case PLFFT_DATA_TYPE_Q15: return 2;
  }
  return 0;
}

// logical element counts of one transform (docs/plfft.md:109-116)
static void io_counts(const ConfigData& c, int64_t& nin, int64_t& nout, bool& in_cplx, bool& out_cplx) {
  const int64_t h = c.n / 2 + 1;
  switch (c.kind) {
    case TKind::C2C: nin = c.n; nout = c.n; in_cplx = out_cplx = true; break;
    case TKind::R2C: nin = c.n; nout = h; in_cplx = false; out_cplx = true; break;
    case TKind::C2R: nin = h; nout = c.n; in_cplx = true; out_cplx = false; break;
    case TKind::R2R: nin = c.n; nout = c.n; in_cplx = out_cplx = false; break;
  }
}

static int64_t span(int64_t howmany, int64_t dist, int64_t n, int64_t stride) {
  return (howmany - 1) * (howmany > 1 ? dist : 0) + (n - 1) * stride + 1;
}

static std::unique_ptr<Node> make_half_node(const ConfigData& c, const Layout& lay, std::string* why);

// plfft_r2r_kind_t -> RealWrapKind
static int r2r_wrap_kind(int payload) {
  static const int map[] = {RW_DCT1, RW_DCT2, RW_DCT3, RW_DCT4, RW_DST1, RW_DST2,
                            RW_DST3, RW_DST4, RW_DHT,  RW_R2HC, RW_HC2R};
  return map[payload];
}

// device schedule for configuration c over the batch layout lay; tune:
// allow plan-time autotuning (rigor above ESTIMATE)
static std::unique_ptr<Node> make_root(const ConfigData& c, const Layout& lay, bool tune, std::string* why,
                                       std::string* note) {
  std::unique_ptr<Node> root;
  const float scale = float(c.scale);
  if (c.data_type == PLFFT_DATA_TYPE_FP32) {
    switch (c.kind) {
      case TKind::C2C:
        if (!tune || c.rigor == PLFFT_ESTIMATE)
          root = make_c2c_node(c.n, lay, c.payload, scale, c.precision, why);
        else
          root = autotune_c2c(c, lay, why, note);
        break;
      case TKind::R2C:
        if (tune && c.rigor != PLFFT_ESTIMATE) {
          root = autotune_real(c, lay, FR_R2C, RW_R2C, why, note);
          break;
        }
        root = make_real_fused_node(FR_R2C, c.n, lay, scale);
        if (!root) root = make_realwrap_node(RW_R2C, c.n, lay, scale, why);
        break;
      case TKind::C2R:
        if (tune && c.rigor != PLFFT_ESTIMATE) {
          root = autotune_real(c, lay, FR_C2R, RW_C2R, why, note);
          break;
        }
        root = make_real_fused_node(FR_C2R, c.n, lay, scale);
        if (!root) root = make_realwrap_node(RW_C2R, c.n, lay, scale, why);
        break;
      case TKind::R2R: {
        if (tune && c.rigor != PLFFT_ESTIMATE) {
          static const int fused_of[] = {-1, FR_DCT2, FR_DCT3, FR_DCT4, -1, FR_DST2,
                                         FR_DST3, FR_DST4, FR_DHT, FR_R2HC, FR_HC2R};
          root = autotune_real(c, lay, fused_of[c.payload], r2r_wrap_kind(c.payload), why, note);
          break;
        }
        if (c.payload == PLFFT_R2R_DCT_2) root = make_real_fused_node(FR_DCT2, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_DST_2) root = make_real_fused_node(FR_DST2, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_DCT_3) root = make_real_fused_node(FR_DCT3, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_DST_3) root = make_real_fused_node(FR_DST3, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_DCT_4) root = make_real_fused_node(FR_DCT4, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_DST_4) root = make_real_fused_node(FR_DST4, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_R2HC) root = make_real_fused_node(FR_R2HC, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_HC2R) root = make_real_fused_node(FR_HC2R, c.n, lay, scale);
        if (c.payload == PLFFT_R2R_DHT) root = make_real_fused_node(FR_DHT, c.n, lay, scale);
        if (!root) root = make_realwrap_node(r2r_wrap_kind(c.payload), c.n, lay, scale, why);
        break;
      }
    }
  } else if (c.data_type == PLFFT_DATA_TYPE_FP64) {
    if (c.precision != 0) {
      if (why) *why = "the split-BF16 precision mode takes FP32 data";
    } else {
      if (c.kind == TKind::R2R)
        root = make_realwrap_node(r2r_wrap_kind(c.payload), c.n, lay, c.scale, why, AW_NONE, AW_NONE, true);
      else
        root = make_fp64_node(int(c.kind), c.n, lay,
                              c.kind == TKind::C2C ? c.payload : (c.kind == TKind::R2C ? -1 : 1), c.scale, why);
    }
  } else if (c.data_type == PLFFT_DATA_TYPE_FP16) {
    if (c.precision != 0) {
      if (why) *why = "the split-BF16 precision mode takes FP32 data";
    } else {
      root = make_half_node(c, lay, why);
    }
  } else if ((c.data_type == PLFFT_DATA_TYPE_Q15 || c.data_type == PLFFT_DATA_TYPE_Q7) &&
             (c.kind == TKind::C2C || c.kind == TKind::R2C || c.kind == TKind::C2R)) {
    if (c.scale != 1.0) {
      if (why) *why = "fixed-point transforms are scaled by 1/n and take no extra scale";
    } else if (c.precision != 0) {
      if (why) *why = "the split-BF16 precision mode takes FP32 data";
    } else {
      root = make_fixed_node(c.data_type == PLFFT_DATA_TYPE_Q15 ? 16 : 8, c.n, lay, c.payload, why,
                             c.kind == TKind::R2C ? 1 : (c.kind == TKind::C2R ? 2 : 0));
    }
  } else if ((c.data_type == PLFFT_DATA_TYPE_Q15 || c.data_type == PLFFT_DATA_TYPE_Q7) &&
             c.kind == TKind::R2R) {
    // fixed-point real-to-real has no implementation (reference src/plfft.cpp:248-261)
    if (why) *why = "fixed-point R2R is not supported";
  } else {
    if (why) *why = "data type not supported on the device path";
  }
  return root;
}

// FP16 (binary16) data: widen a chunk of members into dense FP32, run the
// FP32 schedule for that chunk, round the results back to binary16.
struct HalfIoNode : Node {
  std::unique_ptr<Node> inner, inner_tail;  // FP32 schedules: full chunk, last chunk
  void status_words(std::vector<int*>& out) const override {
    inner->status_words(out);
    if (inner_tail) inner_tail->status_words(out);
  }
  Layout user{};
  int64_t chunk = 1, nin = 0, nout = 0;
  int icomps = 1, ocomps = 1;
  size_t in_bytes() const { return size_t(chunk * nin * icomps) * sizeof(float); }
  size_t out_bytes() const { return size_t(chunk * nout * ocomps) * sizeof(float); }
  size_t inner_ws() const {
    return std::max(inner->workspace(), inner_tail ? inner_tail->workspace() : size_t(0));
  }
  size_t workspace() const override { return (in_bytes() + 255) / 256 * 256 + (out_bytes() + 255) / 256 * 256 + inner_ws(); }
  int launches() const override {
    const int64_t chunks = (user.howmany + chunk - 1) / chunk;
    return int(chunks) * (2 + inner->launches());
  }
  cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const override {
    auto* base = static_cast<unsigned char*>(ws);
    float* din = reinterpret_cast<float*>(base);
    float* dout = reinterpret_cast<float*>(base + (in_bytes() + 255) / 256 * 256);
    void* iws = base + (in_bytes() + 255) / 256 * 256 + (out_bytes() + 255) / 256 * 256;
    for (int64_t m0 = 0; m0 < user.howmany; m0 += chunk) {
      const int64_t cnt = std::min(chunk, user.howmany - m0);
      const Node& node = cnt == chunk ? *inner : *inner_tail;
      cudaError_t e = launch_half_gather(in, din, m0, cnt, nin, user.istride, user.idist, icomps, st);
      if (e == cudaSuccess) e = node.run(din, dout, iws, st);
      if (e == cudaSuccess) e = launch_half_scatter(dout, out, m0, cnt, nout, user.ostride, user.odist, ocomps, st);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  std::string describe() const override {
    return "(fp16 io: binary16 <-> FP32 chunks of " + std::to_string(chunk) + ") + " + inner->describe();
  }
};

static std::unique_ptr<Node> make_half_node(const ConfigData& c, const Layout& lay, std::string* why) {
  int64_t nin = 0, nout = 0;
  bool ic = false, oc = false;
  io_counts(c, nin, nout, ic, oc);
  auto node = std::make_unique<HalfIoNode>();
  node->user = lay;
  node->nin = nin;
  node->nout = nout;
  node->icomps = ic ? 2 : 1;
  node->ocomps = oc ? 2 : 1;
  // in-place: one chunk, so no member's input is overwritten before it is read
  const int64_t per = (nin * node->icomps + nout * node->ocomps) * int64_t(sizeof(float));
  node->chunk = c.alias == PLFFT_IO_MAY_ALIAS
                    ? c.howmany
                    : std::max<int64_t>(1, std::min<int64_t>(c.howmany, (int64_t(256) << 20) / per));
  ConfigData c32 = c;
  c32.data_type = PLFFT_DATA_TYPE_FP32;
  c32.alias = PLFFT_IO_NO_ALIAS;
  const int64_t tail = c.howmany - (c.howmany - 1) / node->chunk * node->chunk;
  std::string note;
  node->inner = make_root(c32, Layout{node->chunk, 1, nin, 1, nout}, false, why, &note);
  if (tail != node->chunk) node->inner_tail = make_root(c32, Layout{tail, 1, nin, 1, nout}, false, why, &note);
  if (!node->inner || (tail != node->chunk && !node->inner_tail)) return nullptr;
  return node;
}

plfft_status_t build_plan(PlanData& p, std::string* why) {
  const ConfigData& c = p.cfg;
  cudaGetDevice(&p.device);
  Layout lay{c.howmany, c.istride, c.howmany > 1 ? c.idist : 0, c.ostride, c.howmany > 1 ? c.odist : 0};
  p.root = make_root(c, lay, true, why, &p.tune_note);
  if (!p.root) return PLFFT_PLAN_CREATION_FAILED;

  int64_t nin = 0, nout = 0;
  bool ic = false, oc = false;
  io_counts(c, nin, nout, ic, oc);
  const int sb = scalar_bytes(c.data_type);
  p.in_bytes = sb * (ic ? 2 : 1);
  p.out_bytes = sb * (oc ? 2 : 1);
  p.nin = nin;
  p.nout = nout;
  p.in_elems = span(c.howmany, c.idist, nin, c.istride);
  p.out_elems = span(c.howmany, c.odist, nout, c.ostride);
  p.out_dense = (c.howmany == 1 && c.ostride == 1) ||
                (c.ostride == 1 && c.odist == nout) ||
                (c.odist == 1 && c.ostride == c.howmany);

  if (p.ws.alloc(p.root->workspace()) != cudaSuccess) {
    if (why) *why = "workspace allocation failed";
    return PLFFT_PLAN_CREATION_FAILED;
  }
  if (cudaStreamCreate(&p.stream) != cudaSuccess) {
    if (why) *why = "stream creation failed";
    return PLFFT_PLAN_CREATION_FAILED;
  }
  return PLFFT_OK;
}

static bool on_device(const void* ptr) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free error of an unknown pointer
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return cudaSuccess;
  return b.alloc(bytes);
}

// Chunked schedules for host-buffer execution, built once (plan mutex held).
// Chunks need members whose spans do not interleave and a dense output.
// (measured on a 64 MiB C2C: chunks of 1 / 2 / 4 / 8 / 16 MiB of traffic
// gave 49 / 53 / 62 / 72 / 73 GB/s end to end)
constexpr int64_t kPipeChunkMb = 16;

static void build_pipe(const PlanData& p) {
  p.pipe_built = true;
  const ConfigData& c = p.cfg;
  const int64_t ib = p.in_elems * p.in_bytes, ob = p.out_elems * p.out_bytes;
  if (c.howmany < 4 || !p.out_dense || c.istride < 1 || c.ostride < 1) return;
  if (c.idist < (p.nin - 1) * c.istride + 1 || c.odist < (p.nout - 1) * c.ostride + 1) return;
  if (ib + ob < (int64_t(16) << 20)) return;  // too small to gain from overlap
  // chunks of about 16 MiB of traffic: the host-to-device copy of chunk i+1,
  // the kernels of chunk i and the device-to-host copy of chunk i-1 overlap
  // (concurrent pinned copies in both directions reach about 95 GB/s)
  int64_t chunk_mb = kPipeChunkMb;
  if (const char* v = std::getenv("PLFFT_B200_PIPE_MB")) chunk_mb = std::max(1, std::atoi(v));
  const int64_t k = std::min<int64_t>(PlanData::kPipeMaxChunks, std::max<int64_t>(2, (ib + ob) / (chunk_mb << 20)));
  const int64_t per = (c.howmany + k - 1) / k;
  const int64_t tail = c.howmany - (c.howmany - 1) / per * per;
  std::string why, note;
  p.pipe_node = make_root(c, Layout{per, c.istride, c.idist, c.ostride, c.odist}, false, &why, &note);
  if (tail != per) p.pipe_tail = make_root(c, Layout{tail, c.istride, c.idist, c.ostride, c.odist}, false, &why, &note);
  if (!p.pipe_node || (tail != per && !p.pipe_tail)) return;
  size_t ws = p.pipe_node->workspace();
  if (p.pipe_tail) ws = std::max(ws, p.pipe_tail->workspace());
  if (p.pipe_ws.alloc(ws) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  for (auto& st : p.pipe_st)
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
  const int64_t chunks = (c.howmany + per - 1) / per;
  for (auto& row : p.pipe_ev)
    for (int64_t i = 0; i < chunks; ++i)
      if (cudaEventCreateWithFlags(&row[i], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return;
      }
  p.pipe_per = per;
}

static cudaError_t execute_pipelined(const PlanData& p, const void* in, void* out) {
  const ConfigData& c = p.cfg;
  const auto* hin = static_cast<const unsigned char*>(in);
  auto* hout = static_cast<unsigned char*>(out);
  auto* din = static_cast<unsigned char*>(p.stage_in.p);
  auto* dout = static_cast<unsigned char*>(p.stage_out.p);
  cudaStream_t s_in = p.pipe_st[0], s_k = p.pipe_st[1], s_out = p.pipe_st[2];
  cudaError_t e = cudaSuccess;
  int i = 0;
  for (int64_t m0 = 0; m0 < c.howmany && e == cudaSuccess; m0 += p.pipe_per, ++i) {
    const int64_t cnt = std::min(p.pipe_per, c.howmany - m0);
    const Node& node = cnt == p.pipe_per ? *p.pipe_node : *p.pipe_tail;
    const size_t ioff = size_t(m0 * c.idist) * p.in_bytes, ooff = size_t(m0 * c.odist) * p.out_bytes;
    const size_t ilen = size_t(span(cnt, c.idist, p.nin, c.istride)) * p.in_bytes;
    const size_t olen = size_t(span(cnt, c.odist, p.nout, c.ostride)) * p.out_bytes;
    e = cudaMemcpyAsync(din + ioff, hin + ioff, ilen, cudaMemcpyHostToDevice, s_in);
    if (e == cudaSuccess) e = cudaEventRecord(p.pipe_ev[0][i], s_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s_k, p.pipe_ev[0][i], 0);
    if (e == cudaSuccess) e = node.run(din + ioff, dout + ooff, p.pipe_ws.p, s_k);
    if (e == cudaSuccess) e = cudaEventRecord(p.pipe_ev[1][i], s_k);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s_out, p.pipe_ev[1][i], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hout + ooff, dout + ooff, olen, cudaMemcpyDeviceToHost, s_out);
  }
  for (auto st : p.pipe_st) {
    const cudaError_t s = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = s;
  }
  return e;
}

plfft_status_t execute_sync(const PlanData& p, const void* in, void* out) {
  std::lock_guard<std::mutex> lock(p.mu);
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != p.device) cudaSetDevice(p.device);
  cudaError_t e = cudaSuccess;
  const bool din = on_device(in), dout = on_device(out);
  const size_t ibytes = size_t(p.in_elems) * p.in_bytes;
  const size_t obytes = size_t(p.out_elems) * p.out_bytes;
  const void* kin = in;
  void* kout = out;
  const uintptr_t i0 = reinterpret_cast<uintptr_t>(in), o0 = reinterpret_cast<uintptr_t>(out);
  const bool overlap = i0 < o0 + obytes && o0 < i0 + ibytes;
  if (!din && !dout && !overlap) {
    if (!p.pipe_built) build_pipe(p);
    if (p.pipe_per > 0) {
      e = ensure(p.stage_in, ibytes);
      if (e == cudaSuccess) e = ensure(p.stage_out, obytes);
      if (e == cudaSuccess) e = execute_pipelined(p, in, out);
      if (cur != p.device) cudaSetDevice(cur);
      if (e != cudaSuccess) return PLFFT_CUDA_ERROR;
      const plfft_status_t a = take_device_status(p.pipe_node.get());
      const plfft_status_t b = take_device_status(p.pipe_tail.get());
      return a != PLFFT_OK ? a : b;
    }
  }
  if (!din) {
    e = ensure(p.stage_in, ibytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p.stage_in.p, in, ibytes, cudaMemcpyHostToDevice, p.stream);
    kin = p.stage_in.p;
  }
  if (e == cudaSuccess && !dout) {
    e = ensure(p.stage_out, obytes);
    // keep the bytes between strided outputs intact
    if (e == cudaSuccess && !p.out_dense)
      e = cudaMemcpyAsync(p.stage_out.p, out, obytes, cudaMemcpyHostToDevice, p.stream);
    kout = p.stage_out.p;
  }
  if (e == cudaSuccess) e = p.root->run(kin, kout, p.ws.p, p.stream);
  if (e == cudaSuccess && !dout) e = cudaMemcpyAsync(out, p.stage_out.p, obytes, cudaMemcpyDeviceToHost, p.stream);
  const cudaError_t s = cudaStreamSynchronize(p.stream);
  if (e == cudaSuccess) e = s;
  if (cur != p.device) cudaSetDevice(cur);
  if (e != cudaSuccess) return PLFFT_CUDA_ERROR;
  // a bounded device wait that ran out leaves its members unwritten
  return take_device_status(p.root.get());
}

}  // namespace plfft_b200
