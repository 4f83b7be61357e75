// Host-side planner and plan objects.
//
// The reference builds a tree of CPU plans (planner strategies in
// src/planner/planner.cpp:49-182, legacy compositor in
// src/compositor.cpp:57-316, level data in src/make_level_data.hpp:100-165)
// and executes it level by level on host memory.  Here the planner picks a
// schedule of device kernels instead: a single on-chip pass when the whole
// transform fits in one CTA's shared memory, a four-step pair of passes for
// longer smooth lengths, and Rader / Bluestein convolutions for lengths with
// large prime factors.  Every node owns its device tables (twiddles, chirps,
// permutations, convolution spectra) and runs asynchronously on a stream.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/plfft.h"
#include "kernels.h"

namespace plfft_b200 {

enum class TKind { C2C = 0, R2C = 1, C2R = 2, R2R = 3 };

// the configuration object behind plfft_config_t
struct ConfigData {
  int64_t n = 0;
  int64_t howmany = 1;
  int64_t istride = 1, idist = 0, ostride = 1, odist = 0;
  TKind kind = TKind::C2C;
  int payload = 0;  // direction for C2C, r2r kind for R2R
  plfft_data_type_t data_type = PLFFT_DATA_TYPE_FP32;
  plfft_io_alias_t alias = PLFFT_IO_NO_ALIAS;
  plfft_sme_mode_t sme = PLFFT_SME_DISABLED;
  plfft_rigor_t rigor = PLFFT_MEASURE;
  // extensions
  double scale = 1.0;
  int precision = 0;  // 0 plain FP32, 1 split-BF16 tensor-core stages
};

// RAII device allocation
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t b) {
    release();
    if (b == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T>
  cudaError_t upload(const std::vector<T>& v) {
    cudaError_t e = alloc(v.size() * sizeof(T));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// One int of pinned host memory mapped into the device's address space: a
// kernel writes a failure code there, the host reads it once the stream that
// ran the kernel has drained (no copy on the success path).
struct HostWord {
  int* p = nullptr;
  HostWord() = default;
  HostWord(const HostWord&) = delete;
  HostWord& operator=(const HostWord&) = delete;
  ~HostWord() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t alloc() {
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&p), sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    *p = 0;
    return cudaSuccess;
  }
  // the address kernels write through (the same address under unified
  // virtual addressing)
  int* device() const {
    void* d = nullptr;
    if (p && cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return static_cast<int*>(d);
  }
};

// Strided batch layout, in elements of the buffer's own type.
struct Layout {
  int64_t howmany;
  int64_t istride, idist, ostride, odist;
};

// One executable piece of a plan.
struct Node {
  virtual ~Node() = default;
  // bytes of device workspace this node needs per execution
  virtual size_t workspace() const { return 0; }
  virtual cudaError_t run(const void* in, void* out, void* ws, cudaStream_t st) const = 0;
  virtual std::string describe() const = 0;
  // number of kernel launches per run (for launch accounting)
  virtual int launches() const { return 1; }
  // host-mapped status words its kernels report device-side failures in
  // (bounded waits that ran out); composite nodes add their parts' words
  virtual void status_words(std::vector<int*>& out) const { (void)out; }
};

// Reads and clears the status words of a node whose kernels have completed:
// PLFFT_DEVICE_TIMEOUT if any reported a failure, else PLFFT_OK.
plfft_status_t take_device_status(const Node* node);

// ---------------------------------------------------------------------------
// factorization and stage tables
// ---------------------------------------------------------------------------
bool is_smooth(int64_t n);  // all prime factors in {2,3,5,7,11,13}
bool is_prime(int64_t n);
std::vector<int> factor_radices(int64_t n, int max_radix);
// builds the stage list and appends the stage twiddle rows to tw
FftDesc make_desc(int n, const std::vector<int>& radices, std::vector<float2>& tw);
// exp(sign * 2 pi i k / n) in double
void unit_root(int64_t k, int64_t n, double& c, double& s);

// largest length one CTA transforms on chip
constexpr int kMaxOnChip = 16384;

// shared-memory tile schedule for length n (c transforms per CTA)
struct TileChoice {
  int maxe = 16, c = 1, nthr = 32, ld = 1;
  std::vector<int> radices;
};
bool choose_tile(int64_t n, bool interleaved, TileChoice& tc);
// four-step split n = n1 * (n / n1) with both factors on chip (0 if none)
int64_t four_step_split(int64_t n);

// C2C FP32 node for a strided batch (dir -1/+1); scale applied on output.
std::unique_ptr<Node> make_c2c_node(int64_t n, const Layout& lay, int dir, float scale,
                                    int precision, std::string* why);

// Alternative C2C schedules for the autotuner, the default first; level 1-3
// widens the search (launch shapes, kernel families, four-step shapes).
std::vector<std::unique_ptr<Node>> make_c2c_candidates(int64_t n, const Layout& lay, int dir, float scale,
                                                       int precision, int level);

// The autotuner's wisdom store (autotune.cpp): problem key -> description
// of the chosen schedule, with the device name for keys
bool wisdom_recall(const std::string& key, std::string& choice);
void wisdom_remember(const std::string& key, const std::string& choice);
std::string wisdom_device();

// Plan-time autotuning for rigor MEASURE/PATIENT/EXHAUSTIVE (autotune.cpp):
// times the candidates and remembers the winner in wisdom; note receives
// "wisdom" or "autotuned k/m candidates".
std::unique_ptr<Node> autotune_c2c(const ConfigData& c, const Layout& lay, std::string* why, std::string* note);

// FP64 nodes (plan_fp64.cpp): kind 0 C2C, 1 R2C, 2 C2R; nullptr (with why)
// when the length or kind has no FP64 schedule.
std::unique_ptr<Node> make_fp64_node(int kind, int64_t n, const Layout& lay, int dir, double scale,
                                     std::string* why);

// Fixed-point C2C (kind 0), R2C (kind 1) or C2R (kind 2) node (plan_fixed.cpp), bits 16
// (Q0.15) or 8 (Q0.7); nullptr (with why) if unsupported.
std::unique_ptr<Node> make_fixed_node(int bits, int64_t n, const Layout& lay, int dir, std::string* why,
                                      int kind = 0);

// FP64 host helpers for table generation (plan_conv.cpp)
using cd = std::complex<double>;
std::vector<cd> host_fft(const std::vector<cd>& x, int sign);
std::vector<float2> to_f2(const std::vector<cd>& v, double scale);
int64_t pow_mod(int64_t a, int64_t e, int64_t p);
int64_t primitive_root(int64_t p);

// Rader (prime n, smooth n-1) or Bluestein (any n) convolution node.
std::unique_ptr<Node> make_conv_node(int64_t n, const Layout& lay, int dir, float scale, std::string* why);
// one-launch Rader / Bluestein when the convolution fits a power-of-two
// length <= 8192 (conv_fused_length(n) != 0); e = 0 picks the default shape
int64_t conv_fused_length(int64_t n);
std::unique_ptr<Node> make_conv_fused(int64_t n, const Layout& lay, int dir, float scale, std::string* why, int e,
                                      int minb, int g);
int64_t next_smooth(int64_t n);

// R2C / C2R / R2R through a C2C plan of a related length (realwrap.cu);
// kind is a RealWrapKind.  fp64: double data around an FP64 C2C plan.
std::unique_ptr<Node> make_realwrap_node(int kind, int64_t n, const Layout& lay, double scale, std::string* why,
                                         int wmode_in = 0, int wmode_out = 0, bool fp64 = false);

// FP64 C2C node (plan_fp64.cpp); nullptr (with why) for lengths without a
// schedule.
std::unique_ptr<Node> make_fp64_c2c(int64_t n, const Layout& lay, int dir, double scale, std::string* why);

// One-kernel R2C / C2R / DCT-II / DST-II (FusedRealKind) for N = 2M, M a
// power of two in [64, 8192], unit strides; nullptr when not applicable.
// wmode: adjoint weights (RealFusedLaunch::wmode), 0 for the plain transform.
std::unique_ptr<Node> make_real_fused_node(int kind, int64_t n, const Layout& lay, float scale, int wmode = 0,
                                           int g_override = 0, int e_override = 0);

// Alternative schedules of a real-data transform (fused kind or -1, the
// real-wrap kind), the default first, for the autotuner.
std::vector<std::unique_ptr<Node>> make_real_candidates(int fused_kind, int wrap_kind, int64_t n, const Layout& lay,
                                                        float scale, int level);

// Plan-time autotuning of a real-data transform (rigor above ESTIMATE):
// times make_real_candidates and remembers the winner in wisdom.
std::unique_ptr<Node> autotune_real(const ConfigData& c, const Layout& lay, int fused_kind, int wrap_kind,
                                    std::string* why, std::string* note);

// Adjoint of a plan's transform (same scale, input/output layouts swapped):
// the conjugate-direction C2C, or the transposed real transform expressed
// as another kind with elementwise weights.
std::unique_ptr<Node> make_adjoint_node(const ConfigData& c, std::string* why);

// The plan object behind plfft_plan_t.
struct PlanData {
  ConfigData cfg;
  std::unique_ptr<Node> root;
  int device = 0;
  DevBuf ws;  // workspace for plfft_plan_execute and *_async without a
              // caller-provided workspace
  // adjoint schedule, built on the first adjoint execution
  mutable std::unique_ptr<Node> adjoint;
  mutable DevBuf adj_ws;
  // host-pointer staging (plfft_plan_execute with host buffers)
  mutable std::mutex mu;
  mutable DevBuf stage_in, stage_out;
  cudaStream_t stream = nullptr;
  int64_t in_elems = 0, out_elems = 0;  // span of one execute, elements
  int in_bytes = 0, out_bytes = 0;      // element sizes
  bool out_dense = false;               // the output span is fully written
  std::string tune_note;                // how the schedule was chosen (rigor > ESTIMATE)
  int64_t nin = 0, nout = 0;            // logical elements per member
  // host-buffer pipeline (plfft_plan_execute on host pointers): the batch in
  // chunks that flow through three streams (host-to-device copies, kernels,
  // device-to-host copies) ordered by one event pair per chunk, so each copy
  // direction streams back to back; built on first use
  static constexpr int kPipeStreams = 3;
  static constexpr int kPipeMaxChunks = 64;
  mutable bool pipe_built = false;
  mutable int64_t pipe_per = 0;  // members per chunk, 0 = no pipeline
  mutable std::unique_ptr<Node> pipe_node, pipe_tail;
  mutable cudaStream_t pipe_st[kPipeStreams] = {};
  mutable cudaEvent_t pipe_ev[2][kPipeMaxChunks] = {};
  mutable DevBuf pipe_ws;
  ~PlanData();
};

}  // namespace plfft_b200
