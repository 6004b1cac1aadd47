/*
 * gpufft_b200.h — C ABI of libgpufft_b200.so, the single-GPU, B200-native
 * (sm_100a) replacement of GPU_FFT's 3D real-to-complex / complex-to-real
 * transform.  Plain C types only: device pointers are void*, CUDA streams are
 * passed as void* (a cudaStream_t; NULL = the legacy default stream).
 *
 * Data layout and semantics are the reference's at procs=1
 * (GPU_FFT/src/GPU_FFT/GPU_FFT.h:111-121, Readme.md:47-52):
 *  - real field: Nx x Ny x 2*(Nz/2+1) reals, row-major, each z-row padded by
 *    2*(Nz/2+1)-Nz cells (GPU_FFT_TEST_SCRIPT/test.cu:124-135);
 *  - spectrum, in place over the same bytes: Nx x Ny x (Nz/2+1) complex
 *    (float2 / double2), kz fastest, ky, then kx — numpy.fft.rfftn's order;
 *  - forward sign exp(-i...), no normalisation: c2r(r2c(f)) = Nx*Ny*Nz*f;
 *  - c2r ignores the imaginary parts of bins kz=0 and kz=Nz/2 (even Nz), and
 *    leaves the padding cells of every real row at zero.
 * Both directions are asynchronous on the given stream (the reference returns
 * with its last cuFFT launch in flight too, FFT_R2C.cu:69) and capturable in a
 * CUDA graph: no host synchronisation, no allocation, no cuFFT.
 *
 * Every call returns a gpufft_status; gpufft_last_error() describes the most
 * recent failure of the calling thread.  Nothing throws across the ABI.
 */
#ifndef GPUFFT_B200_H_
#define GPUFFT_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GPUFFT_FLOAT = 0,  /* float  / cufftComplex       (TRANSITIONS::T1_f, T2_f) */
    GPUFFT_DOUBLE = 1  /* double / cufftDoubleComplex (TRANSITIONS::T1_d, T2_d) */
} gpufft_dtype;

typedef enum {
    GPUFFT_SUCCESS = 0,
    GPUFFT_ERR_INVALID = 1,      /* bad argument (size < 1, null pointer, bad dtype) */
    GPUFFT_ERR_UNSUPPORTED = 2,  /* valid but not handled (procs > 1, odd Nz, prime factor > 13, axis too long) */
    GPUFFT_ERR_CUDA = 3,         /* a CUDA runtime call failed */
    GPUFFT_ERR_NOT_INIT = 4,     /* no plan for this dtype: call gpufft_init first */
    GPUFFT_ERR_OOM = 5,          /* device allocation failed, or a request larger than a server's budget */
    GPUFFT_ERR_TIMEOUT = 6,      /* a bounded wait ran out */
    GPUFFT_ERR_CANCELLED = 7     /* the request was cancelled before it started */
} gpufft_status;

typedef struct gpufft_plan_s *gpufft_plan;

/* --------------------------------------------------------------------------
 * Reference-shaped entry points (one plan per dtype per process).
 * ------------------------------------------------------------------------ */

/* Replaces GPU_FFT::INIT_GPU_FFT<T1,T2>(Nx,Ny,Nz,procs,rank,comm)
 * (GPU_FFT/src/initialize_GPU_FFT/GPU_FFT_init.cu:41-93, with
 * INIT_GPU_FFT_COMM, communications_setup.cu:56-71).  Builds (or rebuilds) the
 * process-wide plan of `dtype` on the current CUDA device.  procs must be 1
 * (rank 0) here; more ranks go through gpufft_init_dist.  Unlike the
 * reference, float and double plans coexist, re-initialising frees the
 * previous plan, and no field-sized scratch buffer is allocated. */
int gpufft_init(int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank);

/* The same with procs > 1 ranks, one GPU each (the reference's MPI case,
 * GPU_FFT_init.cu:41-93 and communications_setup.cu:56-71): a collective of
 * all ranks, given rank 0's NCCL unique id (gpufft_dist_unique_id, below).
 * gpufft_r2c / gpufft_c2r then run the slab-decomposed transform: x-slab
 * [Nx/p][Ny][2(Nz/2+1)] in, y-slab [Nx][Ny/p][Nz/2+1] out (FFT_R2C.cu:41-70).
 * Needs one exchange buffer of the local slab's size (the reference
 * allocates one of the field's size, GPU_FFT_init.cu:50). */
int gpufft_init_dist(int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank, const void *id);

/* Replaces GPU_FFT::GPU_FFT_R2C<T1,T2>(T1*) (FFT_implementation/FFT_R2C.cu:41-70):
 * in-place forward transform of `data` on `stream`. */
int gpufft_r2c(int dtype, void *data, void *stream);

/* Replaces GPU_FFT::GPU_FFT_C2R<T1,T2>(T2*) (FFT_implementation/FFT_C2R.cu:41-70):
 * in-place inverse transform (unnormalised) of `data` on `stream`. */
int gpufft_c2r(int dtype, void *data, void *stream);

/* Frees the process-wide plans (the reference has no counterpart; its INIT
 * leaks, GPU_FFT_init.cu:50,86-91). */
int gpufft_finalize(void);

/* Human-readable description of the calling thread's last error ("" if none). */
const char *gpufft_last_error(void);

/* --------------------------------------------------------------------------
 * Plan objects: any number of grids / precisions per process.  The reference
 * keeps one global plan (GPU_FFT/src/initialize_GPU_FFT/GPU_FFT.cu:41-106);
 * these are what the batched and serving layers build on.
 * ------------------------------------------------------------------------ */
int gpufft_plan_create(gpufft_plan *plan, int64_t nx, int64_t ny, int64_t nz, int dtype);
int gpufft_plan_destroy(gpufft_plan plan);
/* Reads the plan's device-side error flags (synchronous): GPUFFT_ERR_CUDA if
 * a bounded wait inside one of its kernels ran out since the plan was made
 * (the queue-scheduled Pass A waiting for a plane, or the tensor-core x pass
 * waiting for its MMAs; the results of that call are wrong and the plan
 * should be destroyed), else GPUFFT_SUCCESS.  No reference counterpart. */
int gpufft_plan_check(gpufft_plan plan);
int gpufft_exec_r2c(gpufft_plan plan, void *data, void *stream);
int gpufft_exec_c2r(gpufft_plan plan, void *data, void *stream);
/* The same with an epilogue fused into the x pass, for pseudo-spectral steps
 * (the reference leaves normalisation to the caller's own kernel,
 * GPU_FFT_TEST_SCRIPT/test.cu:53-65): every output value is multiplied by
 * `scale` (1.0 = none; 1/(Nx*Ny*Nz) makes C2R the normalised inverse), and
 * with dealias != 0 R2C stores zero for the modes outside the 2/3-rule box
 * |kx| <= Nx/3, |ky| <= Ny/3, kz <= Nz/3.  No extra pass over the field;
 * Nx must be at least 2. */
int gpufft_exec_r2c_ex(gpufft_plan plan, void *data, void *stream, double scale, int dealias);
int gpufft_exec_c2r_ex(gpufft_plan plan, void *data, void *stream, double scale);

/* One of the two kernels of an exec, for per-kernel timing and for callers
 * that fuse their own work between the passes.  pass 0 = Pass A (z and y
 * axes, one x-plane per CTA cluster), pass 1 = Pass B (x axis).  A forward
 * transform is pass 0 then pass 1; an inverse is pass 1 then pass 0.  (The
 * reference's corresponding pieces are its cuFFT 2D R2C/C2R plan and its
 * strided 1D C2C plan, GPU_FFT_init.cu:59-92.) */
int gpufft_exec_pass(gpufft_plan plan, void *data, void *stream, int pass, int forward);

/* --------------------------------------------------------------------------
 * Autotuning and wisdom.  The reference's INIT builds fixed cuFFT plans
 * (GPU_FFT_init.cu:86-91); here a plan chooses among several compiled kernel
 * shapes per pass (radix lists, tile widths, threads per CTA, cluster
 * layouts).  Autotuning times every candidate on a field-sized buffer and
 * keeps the fastest; the choice is remembered per device and grid
 * ("wisdom"), and can be saved to / loaded from a text file.  If the
 * environment variable GPUFFT_AUTOTUNE is set to 1, gpufft_init and
 * gpufft_plan_create autotune; if GPUFFT_WISDOM names a file, plans read it
 * and autotuning appends to it.
 * ------------------------------------------------------------------------ */
#define GPUFFT_PLAN_AUTOTUNE 1
/* FP32 plans only: the x pass runs its radix-16 stages as 16x16 DFT-matrix
 * products on the tensor cores, in one of two forms (the autotuner picks):
 * tcgen05.mma with TF32 operands split into two terms (three products) and
 * FP32 accumulators in tensor memory (Nx = 512, 16-byte-aligned rows), or
 * mma.sync with BF16 operands split into three terms (six products).  Both
 * stay within about 1e-7 relative L2 of the plain FP32 plan.  Compiled for
 * Nx = 512 and 1024; other Nx give GPUFFT_ERR_UNSUPPORTED.  No reference
 * counterpart (GPU_FFT's transforms are cuFFT's). */
#define GPUFFT_PLAN_TC_SPLIT 2

int gpufft_plan_create_ex(gpufft_plan *plan, int64_t nx, int64_t ny, int64_t nz, int dtype, int flags);

/* Times the candidates of both passes on `scratch` (a device buffer of
 * gpufft_field_bytes() bytes whose contents are overwritten; NULL = allocate a
 * temporary one) on `stream`, keeps the fastest, records it in the wisdom.
 * Synchronises the stream. */
int gpufft_plan_autotune(gpufft_plan plan, void *scratch, void *stream);

int gpufft_wisdom_save(const char *path);
int gpufft_wisdom_load(const char *path);

/* No counterpart in the reference.  In-place transform of `data` on
 * `stream` (forward != 0: R2C, else C2R, same layout and results as
 * gpufft_r2c / gpufft_c2r) that allocates no device memory, for callers that
 * cannot call cudaMalloc: a device heap owned by an external allocator,
 * allocation-free sections of a serving loop, pre-partitioned device memory.
 * Its twiddle tables live in a static device array of 192 KiB that every GPU
 * loading the library holds until exit; every axis must be at most 4096
 * (larger grids are rejected with GPUFFT_ERR_UNSUPPORTED).  Every call
 * rewrites that array with a small kernel on `stream` (nothing is copied
 * from the host), so calls that overlap on the GPU race: serialise them.
 * The first call on each device looks up the array's address; make that
 * first call before any stream capture. */
int gpufft_exec_noalloc(int64_t nx, int64_t ny, int64_t nz, int dtype, int forward, void *data, void *stream);

/* --------------------------------------------------------------------------
 * Batches: many independent transforms (any mix of grids, each forward or
 * inverse) in ONE persistent kernel launch fed by a work queue; a spectral
 * solver's per-step set of fields (e.g. 3 velocity C2R + 6 product R2C) is
 * one call.  The reference transforms one grid per call (GPU_FFT_R2C /
 * GPU_FFT_C2R, FFT_R2C.cu:41-70, FFT_C2R.cu:41-70).  `dims` holds n triples
 * (Nx, Ny, Nz); directions[t] is 1 for R2C, 0 for C2R; data[t] are the n
 * in-place fields.  exec_graph captures the launch once into a CUDA graph and
 * replays it (the data pointers may change between calls).  Scratch (queue
 * head, one counter per transform) is owned by the batch.
 * ------------------------------------------------------------------------ */
typedef struct gpufft_batch_s *gpufft_batch;
int gpufft_batch_create(gpufft_batch *batch, int n, const int64_t *dims, const int *directions, int dtype);
int gpufft_batch_destroy(gpufft_batch batch);
int gpufft_batch_exec(gpufft_batch batch, void *const *data, void *stream);
int gpufft_batch_exec_graph(gpufft_batch batch, void *const *data, void *stream);
/* Synchronises `stream`; GPUFFT_ERR_CUDA if an item of the last run gave up
 * waiting for its dependency (bounded wait, about 2 s). */
int gpufft_batch_status(gpufft_batch batch, void *stream);
/* Work items per launch. */
int gpufft_batch_items(gpufft_batch batch);
/* Schedules.  PERSISTENT (the default): the one persistent launch above.
 * BRANCHES: each transform runs its own plan's specialised kernels, the
 * transforms spread over `branches` (1..8) concurrent streams forked from
 * and joined back into the caller's stream (largest field first, each to the
 * least loaded stream); exec_graph captures the fork/join as one CUDA graph
 * (captured again when the data pointers change).  Results are bitwise those
 * of the transforms' own plans. */
#define GPUFFT_BATCH_PERSISTENT 0
#define GPUFFT_BATCH_BRANCHES 1
int gpufft_batch_set_schedule(gpufft_batch batch, int schedule, int branches);
int gpufft_batch_schedule(gpufft_batch batch, int *schedule, int *branches);
/* Tunes every distinct grid's plan (gpufft_plan_autotune), then times the
 * persistent launch and 2, 4 and 8 branches (graph replays on scratch
 * fields it allocates and frees) and keeps the fastest schedule. */
int gpufft_batch_autotune(gpufft_batch batch, void *stream);

/* --------------------------------------------------------------------------
 * Fields in host memory (no counterpart in the reference, whose transforms
 * take device fields, FFT_R2C.cu:41-70): a pipe owns `depth` (1..8) device
 * fields of `plan`'s size and three streams (copy-in, compute, copy-out).
 * Each submission copies host_in to a free device field, runs the op
 * (R2C, C2R, or R2C then C2R) and copies the result to host_out, stream-
 * ordered after `stream` at the time of the call; the copy-in of the next
 * submissions overlaps this one's compute and copy-out (PCIe carries both
 * directions at once).  gpufft_hostpipe_join makes `stream` wait for every
 * submission so far.  Host buffers of gpufft_field_bytes() bytes, pinned for
 * the copies to overlap, untouched until the join.  `plan` must outlive the
 * pipe.
 * ------------------------------------------------------------------------ */
#define GPUFFT_PIPE_C2R 0
#define GPUFFT_PIPE_R2C 1
#define GPUFFT_PIPE_ROUNDTRIP 2
typedef struct gpufft_hostpipe_s *gpufft_hostpipe;
int gpufft_hostpipe_create(gpufft_hostpipe *pipe, gpufft_plan plan, int depth);
int gpufft_hostpipe_submit(gpufft_hostpipe pipe, const void *host_in, void *host_out, int op, void *stream);
int gpufft_hostpipe_join(gpufft_hostpipe pipe, void *stream);
int gpufft_hostpipe_destroy(gpufft_hostpipe pipe);

/* --------------------------------------------------------------------------
 * Precision form (no counterpart in the reference, which is FP32/FP64 only,
 * GPU_FFT.h:112-120): the in-place field is stored in 16 bits — format 0 =
 * BF16, 1 = FP16 — half the bytes of the FP32 form, with one FP32 scale per
 * pencil; butterflies run in FP32.  `scales` is a device buffer of
 * gpufft_plan16_scale_count() floats: per z-row scales of the real field
 * (index x*Ny + y) before R2C / after C2R, per x-pencil scales of the
 * spectrum (index ky*(Nz/2+1) + kz) after R2C / before C2R.  A stored value
 * is value/scale with scale = max(|re|,|im|) over its pencil.  Grids with
 * compiled kernels: cubic 64, 96, 128, 192, 256, 384, 512 and 1024.
 * ------------------------------------------------------------------------ */
typedef struct gpufft_plan16_s *gpufft_plan16;
int gpufft_plan16_create(gpufft_plan16 *plan, int64_t nx, int64_t ny, int64_t nz, int format);
int gpufft_plan16_destroy(gpufft_plan16 plan);
int64_t gpufft_plan16_scale_count(gpufft_plan16 plan);
int gpufft_exec16_r2c(gpufft_plan16 plan, void *data, float *scales, void *stream);
int gpufft_exec16_c2r(gpufft_plan16 plan, void *data, float *scales, void *stream);
/* One kernel of a 16-bit transform (pass 0 = A, 1 = B; forward 1 or 0), as
 * gpufft_exec_pass: forward is A then B, inverse B then A. */
int gpufft_exec16_pass(gpufft_plan16 plan, void *data, float *scales, void *stream, int pass, int forward);
/* FP32 padded real field (Nx*Ny*2*(Nz/2+1) floats) -> 16-bit field + per-row scales. */
int gpufft_quantize16(gpufft_plan16 plan, const float *field, void *data, float *row_scales, void *stream);
/* 16-bit field -> FP32 (spectrum != 0: per x-pencil scales; else per z-row scales). */
int gpufft_dequantize16(gpufft_plan16 plan, const void *data, const float *scales, float *out, int spectrum,
                        void *stream);

/* --------------------------------------------------------------------------
 * Slab decomposition over `procs` GPUs, one process (rank) each — the
 * reference's procs > 1 path: INIT_GPU_FFT with procs/rank/comm
 * (GPU_FFT_init.cu:41-93, communications_setup.cu:56-71) and GPU_FFT_R2C /
 * GPU_FFT_C2R (FFT_R2C.cu:41-70, FFT_C2R.cu:41-70).  Rank r's buffer holds
 * the real x-slab [Nx/p][Ny][2(Nz/2+1)] (planes r*Nx/p ...) before R2C and the
 * spectral y-slab [Nx][Ny/p][Nz/2+1] (ky = r*Ny/p ...) after it, in place; Nx
 * and Ny must be multiples of procs.  The exchange is NCCL (loaded at run
 * time): rank 0 calls gpufft_dist_unique_id, hands the 128 bytes to every rank
 * (MPI_Bcast, torch.distributed, ...), and every rank calls
 * gpufft_dplan_create with its device current (a collective; bounded by
 * GPUFFT_DIST_INIT_TIMEOUT seconds, default 120).  procs = 1 needs no id (given
 * one, the exchange runs through a one-rank NCCL communicator all the same).
 * ------------------------------------------------------------------------ */
typedef struct gpufft_dplan_s *gpufft_dplan;
#define GPUFFT_UNIQUE_ID_BYTES 128
int gpufft_dist_unique_id(void *id);
int gpufft_dplan_create(gpufft_dplan *plan, int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank,
                        const void *id);
int gpufft_dplan_destroy(gpufft_dplan plan);
/* Every rank calls these in the same order (each issues one all-to-all). */
int gpufft_dexec_r2c(gpufft_dplan plan, void *data, void *stream);
int gpufft_dexec_c2r(gpufft_dplan plan, void *data, void *stream);
/* out[5]: first x-plane and x-planes of the real slab, first ky and ky rows of
 * the spectral slab, complex elements of the local buffer. */
int gpufft_dplan_layout(gpufft_dplan plan, int64_t *out);
/* All `procs` ranks in this process on the current device, exchanging by
 * device copies (no NCCL): the same decomposition on one GPU. */
int gpufft_dgroup_create(gpufft_dplan *plans, int64_t nx, int64_t ny, int64_t nz, int dtype, int procs);
/* The exchange schedule of `rank` (replaces the reference's MPI_Isend /
 * MPI_Irecv loop and its chunk transposes, FFT_R2C.cu:48-66 / FFT_C2R.cu:48-66):
 * the copies between the rank's field and its exchange buffer, and the sends
 * and receives to each peer, in the order the slab plans issue them.  Host
 * only (no device needed).  Each op is 10 int64: kind (0 local 2D copy,
 * 1 send, 2 receive), peer, src buffer (0 field, 1 exchange buffer),
 * src offset, src pitch, dst buffer, dst offset, dst pitch, width, rows
 * (bytes).  fused != 0: the plans' Pass A writes / reads the exchange layout
 * itself, so the local copies are left out.  Returns the number of ops, or
 * minus the number needed when `cap` is too small. */
int gpufft_dist_schedule(int64_t nx, int64_t ny, int64_t nz, int dtype, int procs, int rank, int forward, int fused,
                         int64_t *ops, int cap);
int gpufft_dgroup_exec(gpufft_dplan *plans, void **data, int procs, int forward, void *stream);

/* --------------------------------------------------------------------------
 * Serving: a continuous-batching request loop (no counterpart in the
 * reference, which is one call per transform, FFT_R2C.cu:41-70).  Plans,
 * twiddle tables and fields stay resident on the device; a dispatcher thread
 * admits queued requests as stream slots and HBM budget free up, runs them
 * concurrently on its streams and reports latency from submit to completion.
 * ------------------------------------------------------------------------ */
typedef enum { GPUFFT_REQ_F32 = 0, GPUFFT_REQ_F64 = 1, GPUFFT_REQ_BF16 = 2, GPUFFT_REQ_FP16 = 3 } gpufft_req_precision;
typedef enum {
    GPUFFT_REQ_QUEUED = 0,
    GPUFFT_REQ_RUNNING = 1,
    GPUFFT_REQ_DONE = 2,
    GPUFFT_REQ_FAILED = 3,
    GPUFFT_REQ_CANCELLED = 4
} gpufft_req_status;
typedef struct {
    int64_t nx, ny, nz;
    int precision;   /* gpufft_req_precision */
    int direction;   /* 1 = R2C, 0 = C2R */
    void *data;         /* device field, in place */
    float *scales;      /* per-pencil scales (16-bit precisions only) */
    void *ready_event;  /* cudaEvent_t the transform waits for (the producer of
                           the field recorded it), or NULL if the field is
                           already complete when submitted */
} gpufft_request;
typedef struct {
    int64_t completed, failed, cancelled, queued, in_flight, max_in_flight;
    int64_t bytes_in_use, peak_bytes_in_use, plans;
    double p50_ms, p99_ms;
    int64_t records; /* request records held: submitted and not yet released */
} gpufft_server_stats_t;
typedef struct gpufft_server_s *gpufft_server;
#define GPUFFT_SERVER_DRYRUN 1 /* host timers instead of the GPU (tests of the scheduling) */

/* budget_bytes: sum of the field bytes of admitted requests; slots: requests
 * in flight at once (one CUDA stream each). */
int gpufft_server_create(gpufft_server *server, int64_t budget_bytes, int slots, int flags);
/* Stops admitting, lets requests in flight finish, fails those still queued. */
int gpufft_server_stop(gpufft_server server);
int gpufft_server_destroy(gpufft_server server);
/* Builds the plans (one per slot) a request of this shape and precision will
 * use, on the server's device. */
int gpufft_server_prepare(gpufft_server server, const gpufft_request *request);
/* Every submitted request keeps a record (status, latency) until it is
 * released: by gpufft_server_wait once the wait reports its final status, or
 * by gpufft_server_release.  Clients that only poll, or cancel and never
 * wait, release their requests explicitly, or the records accumulate. */
int gpufft_server_submit(gpufft_server server, const gpufft_request *request, int64_t *id);
/* Status and latency; does not release the record. */
int gpufft_server_poll(gpufft_server server, int64_t id, int *status, double *latency_ms);
/* Bounded wait: GPUFFT_ERR_TIMEOUT after timeout_s seconds.  Releases the
 * record when it returns a final status. */
int gpufft_server_wait(gpufft_server server, int64_t id, double timeout_s, double *latency_ms);
/* Releases the record of a request in a final status (done, failed,
 * cancelled); GPUFFT_ERR_INVALID while it is queued or running. */
int gpufft_server_release(gpufft_server server, int64_t id);
int gpufft_server_cancel(gpufft_server server, int64_t id);
int gpufft_server_stats(gpufft_server server, gpufft_server_stats_t *stats);

/* Bytes of the in-place field: Nx*Ny*(Nz/2+1)*sizeof(complex). */
int64_t gpufft_field_bytes(int64_t nx, int64_t ny, int64_t nz, int dtype);

/* Kernel launches one exec issues (for launch accounting). */
int gpufft_plan_launches(gpufft_plan plan);

/* Text description of the plan (radices, tiles, cluster size), NUL-terminated
 * into buf of size len; returns the full length needed. */
int gpufft_plan_describe(gpufft_plan plan, char *buf, int len);

#ifdef __cplusplus
}
#endif

#endif /* GPUFFT_B200_H_ */
