// C-ABI of libplfft_b200.so: the plfft.h functions and the plfft_cuda.h
// extensions.
//
// Config handling and validation follow reference src/plfft.cpp:
//   defaults            :303-319 (FP32, no alias, SME off, rigor MEASURE,
//                        howmany 1, strides 1, distances n)
//   out-param nulling   :306-309, :429-433
//   validation order    :435-486 (null config, size, batch, kind, alias,
//                        SME mode, SME+R2R, SME+fixed point, SME build,
//                        FP16 availability, rigor), then dtype dispatch
//                        :488-513 with fixed-point R2R -> PLAN_CREATION_FAILED
//   status strings      :264-296
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "../../include/plfft.h"
#include "../../include/plfft_cuda.h"
#include "plan.hpp"
#include "plan_kinds.hpp"

using namespace plfft_b200;

struct plfft_config_t {
  ConfigData d;
};
struct plfft_plan_t {
  PlanData p;
};

static thread_local plfft_status_t g_last_status = PLFFT_OK;

static plfft_status_t from_cuda(cudaError_t e) { return e == cudaSuccess ? PLFFT_OK : PLFFT_CUDA_ERROR; }

extern "C" {

const char* plfft_status_to_string(plfft_status_t status) {
  switch (status) {
    case PLFFT_OK: return "success";
    case PLFFT_NULL_ARGUMENT: return "null argument";
    case PLFFT_INVALID_SIZE: return "invalid transform size";
    case PLFFT_UNSUPPORTED_BATCH: return "Unsupported batch or stride configuration";
    case PLFFT_INVALID_TRANSFORM_KIND: return "invalid transform kind";
    case PLFFT_INVALID_DATA_TYPE: return "invalid data type";
    case PLFFT_INVALID_IO_ALIAS: return "invalid I/O alias mode";
    case PLFFT_PLAN_CREATION_FAILED: return "plan creation failed";
    case PLFFT_INVALID_SME_MODE: return "invalid SME mode";
    case PLFFT_SME_NOT_ENABLED: return "SME support was not enabled when building PLFFT";
    case PLFFT_SME_UNSUPPORTED_R2R: return "SME is not supported for real-to-real transforms";
    case PLFFT_FP16_NOT_AVAILABLE: return "native FP16 support is required but unavailable on this CPU";
    case PLFFT_SME_NOT_AVAILABLE: return "SME support is unavailable on this CPU";
    case PLFFT_SME_UNSUPPORTED_FIXED_POINT: return "SME is not supported for fixed-point transforms";
    case PLFFT_INVALID_PLANNER_RIGOR: return "invalid planning rigor level";
    case PLFFT_CUDA_ERROR: return "a CUDA runtime call failed";
    case PLFFT_DEVICE_TIMEOUT: return "a device-side wait timed out";
    case PLFFT_INVALID_ARGUMENT: return "invalid argument";
  }
  return "unknown status";
}

[[noreturn]] static void out_of_memory() {
  std::fputs("Fatal error: out of memory\n", stderr);
  std::abort();
}

static plfft_status_t new_config(plfft_config_t** config, int64_t n, TKind kind, int payload) {
  *config = new (std::nothrow) plfft_config_t;
  if (!*config) out_of_memory();
  ConfigData& d = (*config)->d;
  d.n = n;
  d.howmany = 1;
  d.istride = 1;
  d.idist = n;
  d.ostride = 1;
  d.odist = n;
  d.kind = kind;
  d.payload = payload;
  return PLFFT_OK;
}

static bool valid_direction(int d) { return d == PLFFT_FORWARD || d == PLFFT_BACKWARD; }
static bool valid_r2r(int k) { return k >= PLFFT_R2R_DCT_1 && k <= PLFFT_R2R_HC2R; }

plfft_status_t plfft_config_create(plfft_config_t** config, int64_t n, plfft_direction_t direction) {
  if (!config) return PLFFT_NULL_ARGUMENT;
  *config = nullptr;
  if (!valid_direction(direction)) return PLFFT_INVALID_TRANSFORM_KIND;
  return new_config(config, n, TKind::C2C, int(direction));
}

plfft_status_t plfft_config_create_r2c(plfft_config_t** config, int64_t n) {
  if (!config) return PLFFT_NULL_ARGUMENT;
  *config = nullptr;
  return new_config(config, n, TKind::R2C, PLFFT_FORWARD);
}

plfft_status_t plfft_config_create_c2r(plfft_config_t** config, int64_t n) {
  if (!config) return PLFFT_NULL_ARGUMENT;
  *config = nullptr;
  return new_config(config, n, TKind::C2R, PLFFT_BACKWARD);
}

plfft_status_t plfft_config_create_r2r(plfft_config_t** config, int64_t n, plfft_r2r_kind_t kind) {
  if (!config) return PLFFT_NULL_ARGUMENT;
  *config = nullptr;
  if (!valid_r2r(kind)) return PLFFT_INVALID_TRANSFORM_KIND;
  return new_config(config, n, TKind::R2R, int(kind));
}

void plfft_config_destroy(plfft_config_t* config) { delete config; }

void plfft_config_set_data_type(plfft_config_t* c, plfft_data_type_t v) { c->d.data_type = v; }
plfft_data_type_t plfft_config_get_data_type(const plfft_config_t* c) { return c->d.data_type; }
void plfft_config_set_io_alias(plfft_config_t* c, plfft_io_alias_t v) { c->d.alias = v; }
plfft_io_alias_t plfft_config_get_io_alias(const plfft_config_t* c) { return c->d.alias; }
void plfft_config_set_sme_mode(plfft_config_t* c, plfft_sme_mode_t v) { c->d.sme = v; }
plfft_sme_mode_t plfft_config_get_sme_mode(const plfft_config_t* c) { return c->d.sme; }
void plfft_config_set_rigor(plfft_config_t* c, plfft_rigor_t v) { c->d.rigor = v; }
plfft_rigor_t plfft_config_get_rigor(const plfft_config_t* c) { return c->d.rigor; }
void plfft_config_set_batch(plfft_config_t* c, int64_t howmany, int64_t istride, int64_t idist,
                            int64_t ostride, int64_t odist) {
  c->d.howmany = howmany;
  c->d.istride = istride;
  c->d.idist = idist;
  c->d.ostride = ostride;
  c->d.odist = odist;
}
int64_t plfft_config_get_howmany(const plfft_config_t* c) { return c->d.howmany; }
int64_t plfft_config_get_istride(const plfft_config_t* c) { return c->d.istride; }
int64_t plfft_config_get_idist(const plfft_config_t* c) { return c->d.idist; }
int64_t plfft_config_get_ostride(const plfft_config_t* c) { return c->d.ostride; }
int64_t plfft_config_get_odist(const plfft_config_t* c) { return c->d.odist; }

void plfft_cuda_config_set_scale(plfft_config_t* c, double s) { c->d.scale = s; }
double plfft_cuda_config_get_scale(const plfft_config_t* c) { return c->d.scale; }
void plfft_cuda_config_set_precision(plfft_config_t* c, plfft_cuda_precision_t p) { c->d.precision = int(p); }
plfft_cuda_precision_t plfft_cuda_config_get_precision(const plfft_config_t* c) {
  return plfft_cuda_precision_t(c->d.precision);
}

static bool valid_batch(const ConfigData& d) {
  if (d.howmany == 1) return d.istride > 0 && d.ostride > 0;
  return d.howmany > 0 && d.istride > 0 && d.idist > 0 && d.ostride > 0 && d.odist > 0;
}

static bool valid_kind(const ConfigData& d) {
  switch (d.kind) {
    case TKind::C2C: return valid_direction(d.payload);
    case TKind::R2C:
    case TKind::C2R: return true;
    case TKind::R2R: return valid_r2r(d.payload);
  }
  return false;
}

plfft_status_t plfft_plan_create_from_config(plfft_plan_t** plan, const plfft_config_t* config) {
  if (!plan) return PLFFT_NULL_ARGUMENT;
  *plan = nullptr;
  if (!config) return PLFFT_NULL_ARGUMENT;
  const ConfigData& d = config->d;
  if (d.n <= 0) return PLFFT_INVALID_SIZE;
  if (!valid_batch(d)) return PLFFT_UNSUPPORTED_BATCH;
  if (!valid_kind(d)) return PLFFT_INVALID_TRANSFORM_KIND;
  if (d.alias != PLFFT_IO_NO_ALIAS && d.alias != PLFFT_IO_MAY_ALIAS) return PLFFT_INVALID_IO_ALIAS;
  if (d.sme != PLFFT_SME_DISABLED && d.sme != PLFFT_SME_ENABLED) return PLFFT_INVALID_SME_MODE;
  const bool want_sme = d.sme == PLFFT_SME_ENABLED;
  if (want_sme && d.kind == TKind::R2R) return PLFFT_SME_UNSUPPORTED_R2R;
  if (want_sme && (d.data_type == PLFFT_DATA_TYPE_Q7 || d.data_type == PLFFT_DATA_TYPE_Q15))
    return PLFFT_SME_UNSUPPORTED_FIXED_POINT;
  if (want_sme) return PLFFT_SME_NOT_ENABLED;  // no SME on this target
  if (d.rigor < PLFFT_ESTIMATE || d.rigor > PLFFT_EXHAUSTIVE) return PLFFT_INVALID_PLANNER_RIGOR;
  switch (d.data_type) {
    case PLFFT_DATA_TYPE_FP32:
    case PLFFT_DATA_TYPE_FP64:
    case PLFFT_DATA_TYPE_FP16:
    case PLFFT_DATA_TYPE_Q7:
    case PLFFT_DATA_TYPE_Q15:
      break;
    default:
      return PLFFT_INVALID_DATA_TYPE;
  }
  auto* p = new (std::nothrow) plfft_plan_t;
  if (!p) out_of_memory();
  p->p.cfg = d;
  std::string why;
  const plfft_status_t st = build_plan(p->p, &why);
  if (st != PLFFT_OK) {
    if (std::getenv("PLFFT_B200_VERBOSE")) std::fprintf(stderr, "plfft_b200: %s\n", why.c_str());
    delete p;
    return st;
  }
  *plan = p;
  return PLFFT_OK;
}

void plfft_plan_destroy(plfft_plan_t* plan) {
  if (!plan) return;
  int cur = 0;
  cudaGetDevice(&cur);
  const int dev = plan->p.device;
  if (cur != dev) cudaSetDevice(dev);
  delete plan;
  if (cur != dev) cudaSetDevice(cur);
}

plfft_status_t plfft_cuda_get_last_status(void) { return g_last_status; }

plfft_status_t plfft_cuda_plan_get_workspace_size(const plfft_plan_t* plan, size_t* bytes) {
  if (!plan || !bytes) return PLFFT_NULL_ARGUMENT;
  *bytes = plan->p.root->workspace();
  return PLFFT_OK;
}

int plfft_cuda_plan_get_launch_count(const plfft_plan_t* plan) {
  return plan ? plan->p.root->launches() : 0;
}

plfft_status_t plfft_cuda_plan_describe(const plfft_plan_t* plan, char* buf, size_t len) {
  if (!plan || !buf) return PLFFT_NULL_ARGUMENT;
  std::string s = plan->p.root->describe();
  if (!plan->p.tune_note.empty()) s += " [" + plan->p.tune_note + "]";
  if (len == 0) return PLFFT_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", s.c_str());
  return PLFFT_OK;
}

plfft_status_t plfft_cuda_execute_async(const plfft_plan_t* plan, const void* in, void* out, void* ws,
                                        void* stream) {
  if (!plan || !in || !out) return PLFFT_NULL_ARGUMENT;
  const PlanData& p = plan->p;
  void* w = ws ? ws : p.ws.p;
  const cudaError_t e = p.root->run(in, out, w, static_cast<cudaStream_t>(stream));
  g_last_status = from_cuda(e);
  return g_last_status;
}

plfft_status_t plfft_cuda_plan_get_device_status(const plfft_plan_t* plan, void* stream) {
  if (!plan) return PLFFT_NULL_ARGUMENT;
  const PlanData& p = plan->p;
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) return PLFFT_CUDA_ERROR;
  const plfft_status_t a = take_device_status(p.root.get());
  const plfft_status_t b = take_device_status(p.adjoint.get());
  return a != PLFFT_OK ? a : b;
}

// builds the adjoint schedule once (plan mutex); returns false on failure
static bool ensure_adjoint(const PlanData& p) {
  std::lock_guard<std::mutex> lock(p.mu);
  if (p.adjoint) return true;
  std::string why;
  auto node = make_adjoint_node(p.cfg, &why);
  if (!node) return false;
  if (p.adj_ws.alloc(node->workspace()) != cudaSuccess) return false;
  p.adjoint = std::move(node);
  return true;
}

plfft_status_t plfft_cuda_plan_get_adjoint_workspace_size(const plfft_plan_t* plan, size_t* bytes) {
  if (!plan || !bytes) return PLFFT_NULL_ARGUMENT;
  if (!ensure_adjoint(plan->p)) return PLFFT_PLAN_CREATION_FAILED;
  *bytes = plan->p.adjoint->workspace();
  return PLFFT_OK;
}

plfft_status_t plfft_cuda_execute_adjoint_async(const plfft_plan_t* plan, const void* in, void* out, void* ws,
                                                void* stream) {
  if (!plan || !in || !out) return PLFFT_NULL_ARGUMENT;
  const PlanData& p = plan->p;
  if (!ensure_adjoint(p)) return g_last_status = PLFFT_PLAN_CREATION_FAILED;
  const cudaError_t e = p.adjoint->run(in, out, ws ? ws : p.adj_ws.p, static_cast<cudaStream_t>(stream));
  g_last_status = from_cuda(e);
  return g_last_status;
}

void plfft_plan_execute(const plfft_plan_t* plan, const void* in, void* out) {
  g_last_status = execute_sync(plan->p, in, out);
}

}  // extern "C"
