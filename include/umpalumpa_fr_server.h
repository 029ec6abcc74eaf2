/*
 * umpalumpa_fr_server.h -- serving form of the B200 Fourier-reconstruction engine.
 *
 * No counterpart in the reference, which reconstructs one volume per operation instance:
 * the example driver opens one AFR operation, feeds it projection batches in a loop and
 * reads the volume at the end (examples/fourier_reconstruction/fr.cpp:205-228,
 * fr.hpp:95-151).  A server runs many such reconstructions ("jobs") at once on one GPU:
 *
 *  - a job is opened with its sizes and is ADMITTED when its volume and weights (12 bytes
 *    per voxel) fit in the HBM budget and a job slot is free; jobs that do not fit wait,
 *    first come first served, and are admitted as soon as released jobs free the memory;
 *  - the client streams projection batches into an open job (FFT half-planes plus either
 *    3x3 rotations, from which the server builds the traverse spaces on the GPU, or
 *    ready-made traverse spaces), then closes it;
 *  - a dispatcher thread continuously gathers the pending batches of all admitted jobs
 *    into one batched insertion launch per step (fr_batch_execute), so the work of jobs
 *    that arrived at different times overlaps on the device; staging of the next step's
 *    host-resident inputs and traverse spaces runs on a second stream under the current
 *    step's insertion;
 *  - each job's volume and weights stay in HBM until the client releases the job.
 *
 * Every job's result equals what fr_execute gives for the same batches (insertion only
 * adds, so the result depends on neither the step boundaries nor the other jobs beyond
 * FP32 summation order).
 *
 * Conventions as in umpalumpa_fr.h: FR_OK or a negative FR_E* status, fr_last_error() for
 * the message.  Every function is thread-safe; a job id stays valid until
 * fr_server_release_job, so release a job only after every wait on it or read of it has
 * returned.  A device-side failure (a CUDA error, or a
 * traverse space addressing a projection outside its batch) fails every unfinished job and
 * every later call; destroy the server.
 */
#ifndef UMPALUMPA_FR_SERVER_H
#define UMPALUMPA_FR_SERVER_H

#include "umpalumpa_fr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fr_server fr_server;

typedef struct fr_server_config {
  uint64_t hbm_budget;           /* bytes of job volumes + weights admitted at once          */
  uint64_t staging_bytes;        /* device staging per in-flight step for host-resident FFTs,
                                    scales and rotations (0: 1 GiB)                          */
  uint32_t max_jobs;             /* admitted jobs at once (0: 256)                           */
  uint32_t max_step_projections; /* traverse spaces inserted by one step (0: 65536)          */
  uint32_t max_step_entries;     /* batch slices in one step (0: 256)                        */
  uint32_t max_volume_side;      /* largest volume side of a job (0: 385)                    */
  uint32_t table_elems;          /* blob-table entries for lookup interpolation (0: 10000)   */
  uint32_t pipeline_depth;       /* steps in flight on the GPU, 1 or 2 (0: 2)                */
  uint64_t reserve_bytes;        /* job memory grown into the server's pool at creation and
                                    kept, so admissions within it never wait for the driver
                                    to map new memory (0: none; at most hbm_budget)          */
} fr_server_config;

typedef struct fr_server_job_desc {
  uint32_t fft_x, fft_y;               /* half-plane of every projection [fft_y][fft_x]     */
  uint32_t volume_x, volume_y, volume_z; /* odd, y == z (as fr_init)                        */
  uint32_t image_x, image_y;           /* imgSizeX/Y of the traverse spaces built from
                                          rotations (traverse_space_generator.hpp:94-145)  */
  float space_weight;                  /* TraverseSpace::weight of those spaces (1: as the
                                          reference example, fr.cpp:293-309)                */
} fr_server_job_desc;

/* One batch of projections.  Pointers may be host (pinned or pageable) or device memory;
 * fft and scales must be on the same side.  The caller keeps every buffer valid and
 * unchanged until the batch is done (fr_server_query_job: batches_done > its index). */
typedef struct fr_server_batch {
  const void *fft;                 /* n_projections half-planes in the server's storage type */
  const float *scales;             /* n_projections scales (BF16/FP16 storage), else NULL    */
  const float *rotations;          /* n_projections row-major 3x3 rotations; space i inserts
                                      projection i.  NULL: use `spaces`                       */
  const fr_traverse_space *spaces; /* n_spaces spaces, projectionIndex relative to `fft`     */
  uint64_t n_projections;
  uint64_t n_spaces;               /* ignored when rotations are given                       */
} fr_server_batch;

enum {
  FR_JOB_QUEUED = 0,   /* waiting for HBM budget or a slot                                   */
  FR_JOB_ACTIVE = 1,   /* admitted; volume and weights allocated and zeroed                  */
  FR_JOB_DONE = 2,     /* closed and every batch inserted                                    */
  FR_JOB_FAILED = 3
};

typedef struct fr_server_job_info {
  int32_t state;
  int32_t pad;
  uint64_t batches_submitted;
  uint64_t batches_done;
  uint64_t spaces_done;
  void *volume;          /* device, complex64 [z][y][x]; valid from ACTIVE until release     */
  float *weight;         /* device, float [z][y][x]                                          */
  double t_open;         /* seconds on the server clock (fr_server_clock)                    */
  double t_admit;
  double t_done;
} fr_server_job_info;

typedef struct fr_server_stats {
  uint64_t steps;          /* batched insertion launches                                     */
  uint64_t entries;        /* batch slices inserted                                          */
  uint64_t spaces;         /* traverse spaces inserted                                       */
  uint64_t jobs_done;
  uint64_t bytes_admitted; /* volumes + weights currently held                               */
  uint64_t peak_bytes_admitted;
  uint32_t jobs_active;
  uint32_t jobs_queued;
  uint32_t peak_jobs_active;
  uint32_t pad;
  double busy_ms;          /* GPU time of the steps (CUDA events from staging start to insertion
                              end, time overlapping the previous step counted once)           */
  double max_admit_ms;     /* longest admission of one job (allocating and zeroing its volume) */
} fr_server_stats;

/* Fills `config` with the defaults listed above and a budget of 150 GB. */
void fr_server_config_default(fr_server_config *config);
/* Starts a server on `device`: one batched engine sized by `config`, its blob table (lookup
 * interpolation) built on the GPU, a dispatcher and a completion thread. */
int fr_server_create(int device, const fr_server_config *config, const fr_settings *settings,
                     fr_server **out);
/* Stops the threads after the steps in flight, frees every job and the engine. */
int fr_server_destroy(fr_server *server);
/* Seconds since the server was created (the clock of fr_server_job_info's times). */
double fr_server_clock(const fr_server *server);

/* Opens a job; it is admitted at once if it fits, else queued.  FR_E_CAPACITY if its volume
 * and weights alone exceed the whole budget, FR_E_UNSUPPORTED for sizes the engine rejects. */
int fr_server_open_job(fr_server *server, const fr_server_job_desc *desc, uint64_t *job);
/* Appends a batch to an open job (queued or active).  Never blocks on the GPU. */
int fr_server_submit(fr_server *server, uint64_t job, const fr_server_batch *batch);
/* No more batches: the job is DONE once every submitted batch is inserted. */
int fr_server_close_job(fr_server *server, uint64_t job);
/* Waits until the job is DONE or FAILED (timeout_s < 0: no limit); FR_E_CAPACITY on timeout
 * with `info` (optional) describing the job at that moment. */
int fr_server_wait_job(fr_server *server, uint64_t job, double timeout_s, fr_server_job_info *info);
int fr_server_query_job(fr_server *server, uint64_t job, fr_server_job_info *info);
/* Copies a DONE job's volume (complex64) and weights (float) into caller memory, host or
 * device (either pointer may be NULL). */
int fr_server_read_job(fr_server *server, uint64_t job, void *volume, float *weight);
/* Frees the job's volume and weights (a job must be DONE, FAILED or QUEUED) and admits
 * queued jobs that now fit. */
int fr_server_release_job(fr_server *server, uint64_t job);
int fr_server_get_stats(fr_server *server, fr_server_stats *stats);

/* One retired step, for tracing the request loop (times in seconds on the server clock). */
typedef struct fr_server_step_record {
  double t_formed;    /* the dispatcher picked the step's slices                             */
  double t_enqueued;  /* its staging and insertion were enqueued                             */
  double t_launched;  /* the dispatcher recorded it as in flight                             */
  double t_retired;   /* the completion thread saw it finish                                 */
  float gpu_ms;       /* GPU time of the step not overlapping the previous step (CUDA events) */
  uint32_t slices;    /* batch slices                                                        */
  uint64_t spaces;    /* traverse spaces                                                     */
  uint32_t jobs;      /* distinct jobs                                                       */
  float gpu_span_ms;  /* staging start to insertion end, including time queued behind the
                         previous step                                                       */
} fr_server_step_record;

/* Copies up to `capacity` of the most recently retired steps, oldest first, into `out` and
 * their number into `count`; the server keeps the last 4,096. */
int fr_server_step_log(fr_server *server, fr_server_step_record *out, uint64_t capacity, uint64_t *count);

#ifdef __cplusplus
}
#endif

#endif
