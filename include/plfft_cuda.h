/*
 * plfft_cuda.h -- device-side extensions of the plfft.h API for the B200
 * implementation (libplfft_b200.so).  None of these has a counterpart in the
 * reference's public header; each entry states the reference behaviour it
 * extends.  Streams are passed as `void *` holding a cudaStream_t so that the
 * header needs no CUDA include.
 */
#pragma once

#include <stddef.h>
#include <stdint.h>

#include "plfft.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic used by a plan's FP32 C2C stages (extension of
 * plfft_config_set_data_type).  SPLIT_BF16 evaluates radix-16/32 DFT-matrix
 * stages on tensor cores from bf16 hi/lo splits with FP32 accumulation. */
typedef enum plfft_cuda_precision_t {
  PLFFT_CUDA_PRECISION_FP32 = 0,
  PLFFT_CUDA_PRECISION_SPLIT_BF16 = 1
} plfft_cuda_precision_t;

/* Multiply every output by `scale` (e.g. 1/n for a normalized round trip).
 * Default 1.0: unnormalized, as the reference (docs/plfft.md:121-134).
 * Fixed-point plans ignore it (they always scale by 1/n). */
void plfft_cuda_config_set_scale(plfft_config_t *config, double scale);
double plfft_cuda_config_get_scale(const plfft_config_t *config);

void plfft_cuda_config_set_precision(plfft_config_t *config,
                                     plfft_cuda_precision_t precision);
plfft_cuda_precision_t
plfft_cuda_config_get_precision(const plfft_config_t *config);

/* Status of the calling thread's most recent execute (plfft_plan_execute has
 * no return value, reference include/plfft.h:531). */
plfft_status_t plfft_cuda_get_last_status(void);

/* Bytes of device workspace a plan needs per concurrent execution. */
plfft_status_t plfft_cuda_plan_get_workspace_size(const plfft_plan_t *plan,
                                                  size_t *bytes);

/* Number of kernel launches one execution issues. */
int plfft_cuda_plan_get_launch_count(const plfft_plan_t *plan);

/* Write a one-line description of the plan's device schedule (the analogue
 * of the reference's plan_to_string, include/plfft/fft_plan.hpp:20-36). */
plfft_status_t plfft_cuda_plan_describe(const plfft_plan_t *plan, char *buf,
                                        size_t len);

/* Stream-ordered execution on device pointers.  Returns once the work is
 * enqueued.  `workspace` may be NULL: the plan's own workspace is used, in
 * which case executions of the same plan on different streams must not
 * overlap.  Pass a caller buffer of plfft_cuda_plan_get_workspace_size()
 * bytes to run one plan concurrently on several streams. */
plfft_status_t plfft_cuda_execute_async(const plfft_plan_t *plan,
                                        const void *d_input, void *d_output,
                                        void *d_workspace, void *stream);

/* Device-side failures of earlier stream-ordered executions of this plan.
 * Waits for `stream` to drain, then reports PLFFT_DEVICE_TIMEOUT if any
 * kernel of the plan (or of its adjoint) gave up a bounded wait since the
 * last query -- the members that kernel owned are then unwritten -- and
 * PLFFT_OK otherwise; the report is cleared.  The error convention of
 * plfft_plan_execute (reference include/plfft.h:505-532: void, no checks)
 * leaves no room for it, so the synchronous path reports the same status
 * through plfft_cuda_get_last_status().  Status code from the reference's
 * enum extension PLFFT_DEVICE_TIMEOUT (include/plfft.h of this library). */
plfft_status_t plfft_cuda_plan_get_device_status(const plfft_plan_t *plan,
                                                 void *stream);

/* Adjoint (transpose for real data, conjugate transpose for complex data) of
 * the plan's transform, with the plan's scale: d_input uses the plan's OUTPUT
 * layout and d_output its INPUT layout.  No counterpart in the reference;
 * this is the backward pass used for differentiation (C2C -> opposite
 * direction, R2C <-> C2R with Hermitian-fold weights, DCT-II <-> DCT-III,
 * DST-II <-> DST-III, symmetric kinds self-adjoint).  The adjoint schedule is
 * built on first use.  `d_workspace` may be NULL (plan-owned buffer). */
plfft_status_t plfft_cuda_execute_adjoint_async(const plfft_plan_t *plan,
                                                const void *d_input,
                                                void *d_output,
                                                void *d_workspace,
                                                void *stream);
plfft_status_t
plfft_cuda_plan_get_adjoint_workspace_size(const plfft_plan_t *plan,
                                           size_t *bytes);

/* Grouped execution of many C2C FP32 transforms of different lengths.
 * No counterpart in the reference (a PLFFT user creates one plan per length).
 * Transform i has lengths[i] contiguous complex elements starting at element
 * in_offsets[i] of the input buffer and out_offsets[i] of the output buffer
 * (the output regions must not overlap each other or any input region).
 * Every length is accepted: on-chip lengths, Rader primes, Bluestein lengths
 * and four-step lengths all run inside the same persistent kernel, at most
 * four launches (one per dependency phase) replayed as one CUDA graph. */
typedef struct plfft_cuda_group_t plfft_cuda_group_t;
plfft_status_t plfft_cuda_group_create(plfft_cuda_group_t **group,
                                       int64_t count, const int64_t *lengths,
                                       const int64_t *in_offsets,
                                       const int64_t *out_offsets,
                                       plfft_direction_t direction);
plfft_status_t plfft_cuda_group_execute_async(plfft_cuda_group_t *group,
                                              const void *d_input,
                                              void *d_output, void *stream);
/* plfft_cuda_group_create with a planner rigor (reference include/plfft.h:
 * 192-201 semantics).  PLFFT_ESTIMATE is plfft_cuda_group_create (its
 * default schedule).  MEASURE, PATIENT and EXHAUSTIVE build candidate
 * schedules of the group (four-step tile width, same-length transforms
 * merged into one task, largest radix; 4, 6 and 10 candidates), time each on scratch device buffers of the
 * group's spans within 0.1 / 0.5 / 2 s of timed work, keep the fastest and
 * remember it in the wisdom (plfft_cuda_wisdom_*), keyed by the lengths,
 * offsets, direction and device.  Returns PLFFT_INVALID_PLANNER_RIGOR for
 * other rigor values. */
plfft_status_t plfft_cuda_group_create_tuned(plfft_cuda_group_t **group,
                                             int64_t count,
                                             const int64_t *lengths,
                                             const int64_t *in_offsets,
                                             const int64_t *out_offsets,
                                             plfft_direction_t direction,
                                             plfft_rigor_t rigor);
int plfft_cuda_group_get_launch_count(const plfft_cuda_group_t *group);
plfft_status_t plfft_cuda_group_describe(const plfft_cuda_group_t *group,
                                         char *buf, size_t len);
void plfft_cuda_group_destroy(plfft_cuda_group_t *group);

/* Four-step C2C FP32 transform that allocates no device memory.
 *
 * No counterpart in the reference.  For callers that must not allocate device
 * memory while they run: applications whose framework has already reserved
 * the GPU's memory in its own pool (a cudaMalloc here would fail or fragment
 * that pool), and latency-critical loops where cudaMalloc/cudaFree would
 * synchronize the device.  It needs no plan and no workspace.
 *
 * Layout: `howmany` contiguous transforms of `n` complex FP32 elements (unit
 * stride, distance n) at d_input / d_output (device pointers; in place is
 * allowed); unnormalized, `direction` as in plfft_config_create.  Enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream).
 *
 * Limit: 16384 < n <= 2097152 with every prime factor of n in
 * {2,3,5,7,11,13} and a split n = n1 * n2 with n1, n2 <= 16384; any other n
 * returns PLFFT_INVALID_SIZE.  The scratch is one file-scope device array of
 * 17 MiB (16 MiB intermediate buffer + 1 MiB twiddle tables), held on every
 * GPU that loads the library until the process exits.  The first call on a
 * device, with that device current, looks up the array's address; make that
 * first call before any stream capture begins.  Every call rewrites the
 * parts of the array it reads, and all calls on a device share it, so calls
 * that overlap on the GPU race and must not be issued. */
plfft_status_t plfft_cuda_c2c_execute_noalloc(const void *d_input,
                                             void *d_output, int64_t n,
                                             int64_t howmany,
                                             plfft_direction_t direction,
                                             void *stream);

/* Wisdom: schedules chosen by the MEASURE / PATIENT / EXHAUSTIVE planners,
 * one line per problem ("<problem key>\t<schedule>"), kept per process and,
 * when the environment variable PLFFT_B200_WISDOM names a file, loaded from
 * and appended to that file.  The reference keeps its wisdom private to the
 * process (src/planner/wisdom.hpp:23-37); these persist it explicitly. */
plfft_status_t plfft_cuda_wisdom_export(const char *path);
plfft_status_t plfft_cuda_wisdom_import(const char *path);
void plfft_cuda_wisdom_forget(void);

#ifdef __cplusplus
}
#endif
