/*
 * plfft.h -- configure / plan / execute / destroy API for batched 1D
 * Fourier and real-to-real transforms, executed on an NVIDIA B200 (sm_100a).
 *
 * This header is a drop-in for the PLFFT public interface
 * (include/plfft.h of arm/perf-libs-fft): the same type names, enumerator
 * values and function signatures, so C code written against PLFFT compiles
 * and links against libplfft_b200.so unchanged.  Each declaration below names
 * the reference declaration it replaces.
 *
 * Transform conventions (reference docs/plfft.md:100-134):
 *   forward   X[k] = sum_j x[j] exp(-2 pi i j k / n)
 *   backward  X[k] = sum_j x[j] exp(+2 pi i j k / n)
 * Floating-point transforms are unnormalized; Q0.7/Q0.15 transforms scale by
 * 1/n.  Strides and distances count logical elements of the buffer's own
 * element type: element k of batch member b is at ptr[b*dist + k*stride].
 *
 * Execution model: plfft_plan_execute() accepts either host pointers (the
 * data is staged through device memory and the call returns when the result
 * is back in host memory, exactly like the CPU library) or device pointers
 * (the transform runs on the device and the call returns once it finished).
 * The stream-ordered device entry points are in plfft_cuda.h.
 */
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque configuration (reference include/plfft.h:46). */
typedef struct plfft_config_t plfft_config_t;

/* Opaque plan (reference include/plfft.h:54). */
typedef struct plfft_plan_t plfft_plan_t;

/* Status codes (reference include/plfft.h:57-88); values are identical.
 * Codes >= 100 are device-side conditions this implementation adds. */
typedef enum plfft_status_t {
  PLFFT_OK = 0,
  PLFFT_NULL_ARGUMENT = 1,
  PLFFT_INVALID_SIZE = 2,
  PLFFT_UNSUPPORTED_BATCH = 3,
  PLFFT_INVALID_TRANSFORM_KIND = 4,
  PLFFT_INVALID_DATA_TYPE = 5,
  PLFFT_INVALID_IO_ALIAS = 6,
  PLFFT_PLAN_CREATION_FAILED = 7,
  PLFFT_INVALID_SME_MODE = 8,
  PLFFT_SME_NOT_ENABLED = 9,
  PLFFT_SME_UNSUPPORTED_R2R = 10,
  PLFFT_FP16_NOT_AVAILABLE = 11,
  PLFFT_SME_NOT_AVAILABLE = 12,
  PLFFT_SME_UNSUPPORTED_FIXED_POINT = 13,
  PLFFT_INVALID_PLANNER_RIGOR = 14,
  /* extensions: a CUDA runtime call failed / a device wait ran out */
  PLFFT_CUDA_ERROR = 100,
  PLFFT_DEVICE_TIMEOUT = 101,
  PLFFT_INVALID_ARGUMENT = 102
} plfft_status_t;

/* Direction (reference include/plfft.h:91-96). */
typedef enum plfft_direction_t {
  PLFFT_FORWARD = -1,
  PLFFT_BACKWARD = 1
} plfft_direction_t;

/* Real-to-real kinds, FFTW conventions (reference include/plfft.h:98-134). */
typedef enum plfft_r2r_kind_t {
  PLFFT_R2R_DCT_1 = 0, /* REDFT00, n > 1 */
  PLFFT_R2R_DCT_2 = 1, /* REDFT10 */
  PLFFT_R2R_DCT_3 = 2, /* REDFT01 */
  PLFFT_R2R_DCT_4 = 3, /* REDFT11 */
  PLFFT_R2R_DST_1 = 4, /* RODFT00 */
  PLFFT_R2R_DST_2 = 5, /* RODFT10 */
  PLFFT_R2R_DST_3 = 6, /* RODFT01 */
  PLFFT_R2R_DST_4 = 7, /* RODFT11 */
  PLFFT_R2R_DHT = 8,   /* discrete Hartley transform */
  PLFFT_R2R_R2HC = 9,  /* real -> FFTW half-complex */
  PLFFT_R2R_HC2R = 10  /* FFTW half-complex -> real */
} plfft_r2r_kind_t;

/* Scalar type (reference include/plfft.h:136-154). */
typedef enum plfft_data_type_t {
  PLFFT_DATA_TYPE_FP32 = 0,
  PLFFT_DATA_TYPE_FP64 = 1,
  PLFFT_DATA_TYPE_FP16 = 2,
  PLFFT_DATA_TYPE_Q7 = 3,
  PLFFT_DATA_TYPE_Q15 = 4
} plfft_data_type_t;

/* Input/output overlap permission (reference include/plfft.h:156-172). */
typedef enum plfft_io_alias_t {
  PLFFT_IO_NO_ALIAS = 0,
  PLFFT_IO_MAY_ALIAS = 1
} plfft_io_alias_t;

/* SME request (reference include/plfft.h:174-190).  There is no SME on this
 * target; PLFFT_SME_ENABLED fails plan creation with PLFFT_SME_NOT_ENABLED,
 * as a reference build without SME does. */
typedef enum plfft_sme_mode_t {
  PLFFT_SME_DISABLED = 0,
  PLFFT_SME_ENABLED = 1
} plfft_sme_mode_t;

/* Planner rigor (reference include/plfft.h:192-201).  ESTIMATE takes the
 * planner's first choice; MEASURE and above time candidate schedules on the
 * device (see plfft_cuda.h for the persistent tuning cache). */
typedef enum plfft_rigor_t {
  PLFFT_ESTIMATE = 0,
  PLFFT_MEASURE = 1,
  PLFFT_PATIENT = 2,
  PLFFT_EXHAUSTIVE = 3,
} plfft_rigor_t;

/* reference include/plfft.h:212 */
const char *plfft_status_to_string(plfft_status_t status);

/* reference include/plfft.h:236 -- defaults: FP32, no alias, SME off,
 * rigor MEASURE, howmany 1, strides 1, distances n. */
plfft_status_t plfft_config_create(plfft_config_t **config, int64_t n,
                                   plfft_direction_t direction);
/* reference include/plfft.h:257 */
plfft_status_t plfft_config_create_r2c(plfft_config_t **config, int64_t n);
/* reference include/plfft.h:277 */
plfft_status_t plfft_config_create_c2r(plfft_config_t **config, int64_t n);
/* reference include/plfft.h:297 */
plfft_status_t plfft_config_create_r2r(plfft_config_t **config, int64_t n,
                                       plfft_r2r_kind_t r2r_kind);
/* reference include/plfft.h:308; NULL is a no-op */
void plfft_config_destroy(plfft_config_t *config);

/* Setters store without validation; plan creation validates
 * (reference include/plfft.h:320-425). */
void plfft_config_set_data_type(plfft_config_t *config,
                                plfft_data_type_t precision);
plfft_data_type_t plfft_config_get_data_type(const plfft_config_t *config);
void plfft_config_set_io_alias(plfft_config_t *config, plfft_io_alias_t alias);
plfft_io_alias_t plfft_config_get_io_alias(const plfft_config_t *config);
void plfft_config_set_sme_mode(plfft_config_t *config,
                               plfft_sme_mode_t sme_mode);
plfft_sme_mode_t plfft_config_get_sme_mode(const plfft_config_t *config);
void plfft_config_set_rigor(plfft_config_t *config, plfft_rigor_t rigor);
plfft_rigor_t plfft_config_get_rigor(const plfft_config_t *config);
void plfft_config_set_batch(plfft_config_t *config, int64_t howmany,
                            int64_t istride, int64_t idist, int64_t ostride,
                            int64_t odist);
int64_t plfft_config_get_howmany(const plfft_config_t *config);
int64_t plfft_config_get_istride(const plfft_config_t *config);
int64_t plfft_config_get_idist(const plfft_config_t *config);
int64_t plfft_config_get_ostride(const plfft_config_t *config);
int64_t plfft_config_get_odist(const plfft_config_t *config);

/* reference include/plfft.h:469 -- validation order and status codes follow
 * reference src/plfft.cpp:427-486.  Device tables (twiddles, chirps, Rader
 * spectra) are built here, on the current CUDA device. */
plfft_status_t plfft_plan_create_from_config(plfft_plan_t **plan,
                                             const plfft_config_t *config);
/* reference include/plfft.h:503; NULL is a no-op */
void plfft_plan_destroy(plfft_plan_t *plan);
/* reference include/plfft.h:531 -- host or device pointers; returns when the
 * output is complete.  No status, as in the reference; a CUDA failure is
 * reported by plfft_cuda_get_last_status() (plfft_cuda.h). */
void plfft_plan_execute(const plfft_plan_t *plan, const void *input,
                        void *output);

#ifdef __cplusplus
}
#endif
