/*
 * rcabf.h -- C ABI of librcabf, a B200 (sm_100a) row-column-array (RCA)
 * delay-and-sum I/Q beamformer.
 *
 * Plain C: pointers, sizes and status codes only.  Device buffers are raw
 * CUDA device pointers owned by the caller; streams are passed as void*
 * (a cudaStream_t, NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.m        the wrapper
 *   MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu:103   the kernel
 * Each entry point below names the lines it stands in for.
 */
#ifndef RCABF_H
#define RCABF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RCABF_ABI_VERSION 2

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
/* Codes 1..29 correspond one-to-one to the error identifiers raised by the
 * reference wrapper bfVirtualSourceGeneric_RCA.m (line of the error() call in
 * brackets).  rcabf_status_string() returns "bfVirtualSourceGeneric_RCA:<id>"
 * for those, so callers can report the reference identifier. */
typedef enum rcabf_status {
    RCABF_OK = 0,
    RCABF_ERR_DATA_NOT_NUMERIC = 1,            /* :dataNotNumeric [140] */
    RCABF_ERR_OPTIONS_NOT_STRUCT = 2,          /* :OptionsNotStruct [156] */
    RCABF_ERR_INTERPOLATION_INVALID = 3,       /* :flagInterpolationLanczosInvalid [168] */
    RCABF_ERR_COMPOUNDING_INVALID = 4,         /* :flagCompoundingInvalid [177] */
    RCABF_ERR_MASK_TRANSMIT_INVALID = 5,       /* :flagMaskTransmitInvalid [186] */
    RCABF_ERR_DECREASE_FACTOR_INVALID = 6,     /* :decreaseFactorGPUInvalid [196] */
    RCABF_ERR_GRID_MISSING = 7,                /* :gridBfMissing [209] */
    RCABF_ERR_GRID_INVALID = 8,                /* :gridBfInvalid [223] */
    RCABF_ERR_POS_ELE_MISSING = 9,             /* :posEleMissing [234] */
    RCABF_ERR_POS_ELE_INVALID = 10,            /* :posEleInvalid [248] */
    RCABF_ERR_APERTURE_X_INVALID = 11,         /* :apertureXInvalid [265] */
    RCABF_ERR_APERTURE_Y_INVALID = 12,         /* :apertureYInvalid [284] */
    RCABF_ERR_APERTURE_Z_INVALID = 13,         /* :apertureZInvalid [303] */
    RCABF_ERR_TRANSMIT_NOT_STRUCT = 14,        /* :TransmitNotStruct [313] */
    RCABF_ERR_THETA_OR_VS_REQUIRED = 15,       /* :ThetaORVirtualSourceRequired [326] */
    RCABF_ERR_TILTS_NOT_SAME_LENGTH = 16,      /* :tiltsNotSameLength [341] */
    RCABF_ERR_VS_NOT_SAME_LENGTH = 17,         /* :virtualSourcesNotSameLength [356] */
    RCABF_ERR_THETA_OR_VS_INVALID = 18,        /* :ThetaORVirtualSourceInvalid [366] */
    RCABF_ERR_FLAG_RECEIVE_X_INVALID = 19,     /* :flagReceiveXInvalid [378] */
    RCABF_ERR_PARAM_NOT_STRUCT = 20,           /* :ParamNotStruct [386] */
    RCABF_ERR_FS_MISSING = 21,                 /* :samplingFrequencyMissing [393] */
    RCABF_ERR_FS_INVALID = 22,                 /* :samplingFrequencyInvalid [399] */
    RCABF_ERR_FD_MISSING = 23,                 /* :demodulationFrequencyMissing [406] */
    RCABF_ERR_FD_INVALID = 24,                 /* :demodulationFrequencyInvalid [412] */
    RCABF_ERR_SPEED_OF_SOUND_INVALID = 25,     /* :speedOfSoundInvalid [426] */
    RCABF_ERR_START_TIME_INVALID = 26,         /* :startTimeInvalid [440, 454] */
    /* Codes of this library (no reference counterpart). */
    RCABF_ERR_INVALID_ARGUMENT = 100,  /* NULL pointer, bad enum, bad struct_size */
    RCABF_ERR_SHAPE_MISMATCH = 101,    /* data/output sizes inconsistent with geometry */
    RCABF_ERR_UNSUPPORTED = 102,       /* valid request this build does not implement */
    RCABF_ERR_WORKSPACE_TOO_SMALL = 103,
    RCABF_ERR_OOM_ADMISSION = 104,     /* request larger than the server's HBM budget */
    RCABF_ERR_TIMEOUT = 105,           /* deadline passed before completion */
    RCABF_ERR_CUDA = 106,              /* a CUDA runtime call failed */
    RCABF_ERR_BOUNDS = 107,            /* device-side bound check tripped (never expected) */
    RCABF_ERR_BAD_HANDLE = 108,
    RCABF_ERR_CANCELLED = 109,
    RCABF_ERR_BUSY = 110,              /* server queue full */
    RCABF_ERR_PENDING = 111            /* poll: request not finished yet */
} rcabf_status;

const char *rcabf_status_string(int status);
int rcabf_abi_version(void);
/* Detail of the calling thread's last RCABF_ERR_CUDA: the failing step and
 * CUDA's error string ("" if none).  No reference counterpart. */
const char *rcabf_last_error(void);

/* ------------------------------------------------------------------------ */
/* Enumerations                                                              */
/* ------------------------------------------------------------------------ */
typedef enum rcabf_interp {
    RCABF_INTERP_QUAD3 = 0,   /* reference default, 3-tap quadratic (RCA.cu:355-365) */
    RCABF_INTERP_REF6 = 1,    /* reference "Lanczos 5-lobes": sinc(x)sinc(x/2), 6 taps (RCA.cu:331-350) */
    RCABF_INTERP_LANCZOS = 2  /* Lanczos-a: sinc(x)sinc(x/a), 2a taps, a = lanczos_a (2..4) */
} rcabf_interp;

typedef enum rcabf_table_mode {
    RCABF_TABLES_EXACT = 0,     /* delays built in FP64 on the host, stored as FP32
                                   fractional sample indices + unit phasors */
    RCABF_TABLES_REF_COMPAT = 1 /* reference FP32 arithmetic, operation for operation
                                   (transmit delay RCA.cu:256-269 with its cancellation) */
} rcabf_table_mode;

typedef enum rcabf_grid_kind {
    RCABF_GRID_RECTILINEAR = 0, /* voxel (iz, ix, iy) at (grid_x[ix], grid_y[iy], grid_z[iz]) */
    RCABF_GRID_POINTS = 1       /* n_pix arbitrary points (grid_x/y/z have n_pix entries) */
} rcabf_grid_kind;

typedef enum rcabf_iq_dtype {
    RCABF_IQ_C64 = 0,       /* complex64: float (re, im) pairs */
    RCABF_IQ_C32 = 1,       /* complex32: half (re, im) pairs */
    RCABF_IQ_BF16X2 = 2,    /* bfloat16 (re, im) pairs */
    RCABF_IQ_RF_F32 = 3     /* real float32, I/Q interleaved with Q negated:
                               IQ(n) = RF(2n) - i*RF(2n+1) (RCA.m:475-477) */
} rcabf_iq_dtype;

typedef enum rcabf_storage {
    RCABF_STORE_F32 = 0,   /* complex64 samples in HBM */
    RCABF_STORE_F16 = 1,   /* half (re, im) in HBM, FP32 arithmetic */
    RCABF_STORE_BF16 = 2   /* bfloat16 (re, im) in HBM, FP32 arithmetic */
} rcabf_storage;

typedef enum rcabf_kernel {
    RCABF_KERNEL_AUTO = 0,  /* fused tiled kernel */
    RCABF_KERNEL_FUSED = 1, /* persistent voxel-tiled shared-memory gather, all frames in one launch;
                               voxel-blocked along the steering axis when the geometry allows */
    RCABF_KERNEL_PLAIN = 2, /* one launch per frame, one thread per voxel, global gathers */
    RCABF_KERNEL_FUSED_NOBLOCK = 3, /* the fused kernel with one voxel per thread */
    /* the voxel-blocked fused kernel with a given accumulator store
       (RCABF_ERR_UNSUPPORTED where the geometry allows no voxel blocking):
       tensor memory (sm_100a TMEM) or registers */
    RCABF_KERNEL_FUSED_TMEM = 4,
    RCABF_KERNEL_FUSED_REGS = 5,
    /* the tensor-core kernel (sm_100a tcgen05.mma: each (tx, element) step of
       a 128-voxel tile is a banded product of the voxels' interpolation
       weights with the sample window of all frames of a block, accumulated
       in tensor memory over the acquisition): FP16 or BF16 storage, exact
       tables, compounded output, rectilinear grids, at least 32 frames
       (frame blocks up to 208).  Weights enter the MMA in the storage's
       type as a value plus its remainder (~22 bits in FP16, ~16 in BF16;
       products exact, sums FP32) -- or, with _FP16W (FP16 storage only), as
       one FP16 value (~11 bits, half the tensor work) */
    RCABF_KERNEL_FUSED_TC = 6,
    RCABF_KERNEL_FUSED_TC_FP16W = 7
} rcabf_kernel;

/* ------------------------------------------------------------------------ */
/* Geometry: the probe, the voxel grid, the transmits and the parameters     */
/* ------------------------------------------------------------------------ */
/* Fields mirror the reference structs Geometry / Transmit / Param / Options
 * (bfVirtualSourceGeneric_RCA.m:24-58).  Coordinates in metres, times in
 * seconds, frequencies in hertz, angles in radians. */
typedef struct rcabf_geometry_desc {
    int32_t struct_size;          /* sizeof(rcabf_geometry_desc) */
    int32_t receive_x;            /* Transmit.flagReceiveX: 1 receive on X (column) elements */
    /* receive elements, as given: the library centres them (RCA.m:500-502) */
    int64_t n_ele;
    const double *pos_ele_x, *pos_ele_y, *pos_ele_z;
    /* apertures; NaN = element span after centring (RCA.m:505-521) */
    double aperture_x, aperture_y, aperture_z;
    /* voxel grid */
    int32_t grid_kind;            /* rcabf_grid_kind */
    int32_t reserved0;
    int64_t n_z, n_x, n_y;        /* RECTILINEAR: axis lengths; POINTS: n_z = n_pix, n_x = n_y = 1 */
    const double *grid_x, *grid_y, *grid_z; /* axis coordinates or per-point coordinates */
    int64_t stride_z, stride_x, stride_y;   /* output pixel index = iz*stride_z + ix*stride_x + iy*stride_y */
    /* transmits: tilt angles (converted to virtual sources 10 m behind the
       array, RCA.m:527-541) or virtual sources */
    int64_t n_tx;
    int32_t use_theta;
    int32_t reserved1;
    const double *theta_x, *theta_y;
    const double *vs_x, *vs_y, *vs_z;
    /* Param */
    double fs;                    /* samplingFrequency of the I/Q data */
    double fd;                    /* demodulationFrequency */
    double c;                     /* speedOfSound */
    double t0;                    /* startTime */
    double fnumber;
    /* Options */
    int32_t interp;               /* rcabf_interp */
    int32_t lanczos_a;            /* RCABF_INTERP_LANCZOS: 2..4 */
    int32_t table_mode;           /* rcabf_table_mode */
    int32_t mask_transmit;        /* Options.flagMaskTransmit (RCA.cu:190-219) */
    /* optional receive aberration law (s), added to the receive delay:
       per element (Hyp1_save/..._ab_1.cu:306-311) or per (tx, element)
       (Hyp2/..._ab_2.cu:306-311).  NULL = none. */
    const double *ab_law;
    int32_t ab_per_tx;
    int32_t reserved2;
} rcabf_geometry_desc;

typedef struct rcabf_geometry rcabf_geometry;

/* Builds the delay/apodisation tables for one probe + grid + transmit set and
 * keeps them resident on the current device.  Replaces the per-call host
 * preprocessing of bfVirtualSourceGeneric_RCA.m:459-636 (scalar casts,
 * centring, apertures, virtual sources and their minimum distance to the
 * array) and the per-thread delay arithmetic of RCA.cu:255-311.
 * The stream orders the table uploads; the handle is usable on any stream
 * of the same device after the stream has reached this point. */
int rcabf_create_geometry(const rcabf_geometry_desc *desc, void *stream, rcabf_geometry **out);
int rcabf_destroy_geometry(rcabf_geometry *g);

/* Number of pixels / transmits / receive elements of a geometry. */
int rcabf_geometry_info(const rcabf_geometry *g, int64_t *n_pix, int64_t *n_tx, int64_t *n_ele);

/* Virtual sources and minimum distance to the array the geometry derived
 * (RCA.m:527-558), for inspection; arrays of n_tx doubles, any may be NULL. */
int rcabf_geometry_sources(const rcabf_geometry *g, double *vs_x, double *vs_y, double *vs_z,
                           double *min_dist);

/* ------------------------------------------------------------------------ */
/* Beamforming                                                               */
/* ------------------------------------------------------------------------ */
typedef struct rcabf_beamform_args {
    int32_t struct_size;          /* sizeof(rcabf_beamform_args) */
    int32_t iq_dtype;             /* rcabf_iq_dtype */
    const void *iq;               /* device: [frame][tx][channel][sample] */
    int64_t n_sample;             /* I/Q samples per channel (RF_F32: real samples / 2) */
    int64_t n_ch, n_tx, n_frame;
    int32_t storage;              /* rcabf_storage */
    int32_t compound;             /* Options.flagCompounding: 1 sum over transmits */
    void *out;                    /* device complex64: [frame][compound ? 1 : n_tx][pixel]
                                     ([element][frame][tx][pixel] with per_channel) */
    float *mask;                  /* device float: [compound ? 1 : n_tx][pixel]; may be NULL */
    int32_t accumulate;           /* 1: add into out and mask instead of overwriting */
    int32_t kernel;               /* rcabf_kernel */
    void *workspace;              /* device scratch, >= rcabf_beamform_workspace_size() */
    size_t workspace_bytes;
    int32_t frames_per_block;     /* 0 = automatic */
    int32_t reserved0;
    /* NULL, or 5 cudaEvent_t the call records on `stream` before the ingest,
       after the ingest, after the window-range tables, after the main kernel
       and after the mask kernel (per-stage device timing) */
    void *const *stage_events;
    /* 1: one output per receive element instead of their sum, out laid out
       [element][frame][tx][pixel] (the reference's no-sum kernel,
       NoSum/bfVirtualSourceGeneric_RCA_Nosum.cu:228-229, 275-278, 376-383);
       needs compound = 0; runs the one-frame kernel */
    int32_t per_channel;
    int32_t reserved1;
} rcabf_beamform_args;

/* Scratch bytes rcabf_beamform needs for these arguments. */
int rcabf_beamform_workspace_size(const rcabf_geometry *g, const rcabf_beamform_args *a, size_t *bytes);

/* The launch plan rcabf_beamform would use for these arguments, as a JSON
 * object (kernel, frames per block, tile, window rows, shared memory,
 * workspace) written into buf (NUL-terminated, truncated to len). */
int rcabf_describe_plan(const rcabf_geometry *g, const rcabf_beamform_args *a, char *buf, size_t len);

/* Beamforms every frame and transmit of one acquisition.  Replaces the
 * chunked feval/gather loop of bfVirtualSourceGeneric_RCA.m:640-711 and the
 * kernel bfVirtualSourceGeneric_RCA (RCA.cu:103-390).  Asynchronous on
 * `stream`; no host synchronisation, no allocation. */
int rcabf_beamform(const rcabf_geometry *g, const rcabf_beamform_args *a, void *stream);

/* Beamforms n independent acquisitions in one persistent launch (all must
 * share interp, storage and frames_per_block). */
int rcabf_beamform_batch(int n, const rcabf_geometry *const *g, const rcabf_beamform_args *a,
                         void *stream);

/* rcabf_beamform with the channel data (a->iq) and the output (a->out) in
 * HOST memory, page-locked for the copies to overlap (cudaHostAlloc /
 * cudaHostRegister): the frames go through in chunks of frames_per_chunk
 * (0: about four chunks of whole frame blocks, the last the shortest), each
 * chunk copied in on a copy stream, beamformed on `stream` and copied out on
 * another, so that the copies of one chunk overlap the beamforming of its
 * neighbours and only the first copy in and the last copy out are exposed.
 * Same results as rcabf_beamform on device copies of the buffers.
 * a->workspace: device scratch of rcabf_beamform_host_workspace_size bytes
 * (two chunks of channel data and of output, and one chunk's beamform
 * workspace); a->mask stays a device pointer (computed with the first
 * chunk); accumulate = 1 reads each output chunk in before adding to it;
 * per_channel output is RCABF_ERR_UNSUPPORTED (not frame-major).
 * Asynchronous on `stream`: the output is in host memory, and the host
 * buffers free, once `stream` reaches this call.  Replaces the reference's
 * per-chunk host/device round trip (bfVirtualSourceGeneric_RCA.m:664-711:
 * gpuArray upload, feval, gather), which serialises copies and kernels. */
int rcabf_beamform_host_workspace_size(const rcabf_geometry *g, const rcabf_beamform_args *a,
                                       int32_t frames_per_chunk, size_t *bytes);
int rcabf_beamform_host(const rcabf_geometry *g, const rcabf_beamform_args *a, int32_t frames_per_chunk,
                        void *stream);

/* Size of the static device workspace of rcabf_beamform_noalloc (64 MiB). */
#define RCABF_NOALLOC_WORKSPACE_BYTES ((size_t)64 << 20)

/* rcabf_beamform through the fused kernel with a workspace that is a static
 * device array of RCABF_NOALLOC_WORKSPACE_BYTES instead of a caller buffer
 * (a->workspace and a->workspace_bytes are ignored): the call allocates no
 * device memory.  It is for callers that may not call cudaMalloc: an
 * acquisition loop that must not stall (cudaMalloc can synchronise the
 * device), a host framework that owns the device memory pool (MATLAB's
 * gpuArray allocator, a caching allocator that must see every allocation),
 * or a plugin with no allocator of its own.  The array is held by every GPU
 * that loads the library until the process exits.  No counterpart in the
 * reference, whose wrapper allocates its outputs per call.  The first call
 * on each device looks up the static array's
 * address with that device current and clears the array's error counter (a
 * synchronous step): make it before any stream capture.  Rejected with
 * RCABF_ERR_WORKSPACE_TOO_SMALL (detail in rcabf_last_error()) when the plan
 * needs more than RCABF_NOALLOC_WORKSPACE_BYTES, and with
 * RCABF_ERR_UNSUPPORTED when the plan is the plain kernel.  All calls on one
 * device share the array: calls that overlap in time (other streams, other
 * threads) race and must be serialised by the caller.  Each call checks
 * that the geometry's device is the current device (RCABF_ERR_INVALID_ARGUMENT
 * otherwise).  The looked-up addresses are kept for the life of the process:
 * do not call cudaDeviceReset while the library is loaded. */
int rcabf_beamform_noalloc(const rcabf_geometry *g, const rcabf_beamform_args *a, void *stream);

/* What rcabf_autotune chose for a geometry, frame count and storage. */
typedef struct rcabf_tune_result {
    int32_t struct_size;          /* sizeof(rcabf_tune_result) */
    int32_t voxel_blocked;        /* 0: one voxel per thread; the voxel-blocked kernel with its
                                     accumulators in 1: registers, 2: tensor memory */
    int32_t frames_per_block;
    int32_t tile_u, tile_v, tile_z;   /* voxels per tile along the receive axis, steering axis, depth */
    int32_t window_rows;          /* sample rows staged per step (the shared-memory window depth) */
    int32_t candidates;           /* launch choices timed */
    double best_ms, default_ms;   /* per call: the chosen one, the planner's own */
    int32_t tensor_core;          /* 1: the choice is the tensor-core kernel (RCABF_KERNEL_FUSED_TC) */
    int32_t reserved;
} rcabf_tune_result;

/* Times the fused kernel's launch choices (tile shape, hence window depth,
 * frame block, kernel family -- the tensor-core kernel with hi + remainder
 * weights included where it applies; never the single-FP16-weight variant,
 * which is chosen by name only) on these arguments and keeps the fastest for
 * this geometry, frame count and storage: later calls with
 * frames_per_block = 0 (or the chosen block) plan with it.  No counterpart
 * in the reference, whose launch shape is fixed (RCA.m:640-650).
 * Synchronous; allocates its own scratch; overwrites a->out (a->mask and
 * a->accumulate are ignored).  iters: timed calls per candidate (1..100). */
int rcabf_autotune(const rcabf_geometry *g, const rcabf_beamform_args *a, void *stream, int iters,
                   rcabf_tune_result *res);

/* ------------------------------------------------------------------------ */
/* Serving: continuous batching of requests on one device                    */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference, which beamforms one synchronous call at a
 * time (RCA.m:664-711).  A server owns an HBM arena (the admission budget),
 * a set of streams (launch slots) and a scheduler thread.  Requests name
 * caller-owned device buffers and a geometry handle, which must stay valid
 * until the request completes; their workspace comes from the arena.
 * Requests are admitted in arrival order as slots and arena space free up;
 * queued requests whose plans run the same kernel variant are fused into one
 * persistent launch.  A request whose output or mask is written by a launch
 * in flight, or by an earlier queued request, waits for it, so requests that
 * accumulate into one buffer apply in arrival order. */
typedef struct rcabf_server rcabf_server;

typedef struct rcabf_server_config {
    int32_t struct_size;          /* sizeof(rcabf_server_config) */
    int32_t device;               /* CUDA device ordinal */
    size_t hbm_budget_bytes;      /* workspace arena, allocated once at creation */
    int32_t n_streams;            /* launch slots in flight at once (1..64) */
    int32_t max_queue;            /* queued requests beyond which submit returns RCABF_ERR_BUSY */
    int32_t max_batch;            /* requests fused into one launch (1..24) */
    int32_t batch_window_us;      /* with the device idle, wait this long after an arrival for
                                     more requests to fuse (0 = launch at once) */
} rcabf_server_config;

typedef struct rcabf_server_stats {
    int32_t struct_size;          /* sizeof(rcabf_server_stats) */
    int32_t reserved;
    int64_t submitted, completed, rejected, launches, in_flight, queued;
    double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;   /* submit -> completion, host clock */
    double units_done;            /* nominal voxel.rx.tx.frame units of completed requests */
    double busy_s;                /* time with at least one launch in flight */
    double span_s;                /* first submit -> last completion */
    size_t arena_bytes, arena_peak_bytes;
} rcabf_server_stats;

/* Creates a server: allocates the arena on cfg->device (RCABF_ERR_OOM_ADMISSION
 * if it does not fit) and starts the scheduler thread. */
int rcabf_server_create(const rcabf_server_config *cfg, rcabf_server **out);
/* Queues one request (a copy of *a; its workspace fields are ignored) and
 * returns its ticket without waiting.  RCABF_ERR_OOM_ADMISSION when the plan's
 * workspace is larger than the whole arena, RCABF_ERR_BUSY when the queue is
 * full, plus rcabf_beamform's argument errors. */
int rcabf_server_submit(rcabf_server *s, const rcabf_geometry *g, const rcabf_beamform_args *a, uint64_t *ticket);
/* RCABF_ERR_PENDING while the request runs; RCABF_OK once it is done, with its
 * own status in *status (the ticket is then released). */
int rcabf_server_poll(rcabf_server *s, uint64_t ticket, int *status);
/* As poll, but waits up to timeout_s seconds; RCABF_ERR_TIMEOUT if the request
 * is still running then. */
int rcabf_server_wait_for(rcabf_server *s, uint64_t ticket, double timeout_s, int *status);
int rcabf_server_get_stats(rcabf_server *s, rcabf_server_stats *st);
/* Runs the queued requests to completion, then frees the arena and streams. */
int rcabf_server_destroy(rcabf_server *s);

/* ------------------------------------------------------------------------ */
/* Simulator (the producer of channel data)                                  */
/* ------------------------------------------------------------------------ */
/* Element field of the frequency-domain simulator: for every frequency f,
 * scatterer s and element e, the sum over the element's sub-elements of
 * Green's function x azimuth directivity x elevation directivity (flat, or
 * the 4-Gaussian focused-element model when the elevation focus is within
 * 10 m) x the lens delay phase.  out: device complex64 [n_f][n_scat][n_ele];
 * r_scat: device float [3][n_scat] (x, y, z, metres); r_ele: device float
 * [n_sub][5][n_ele] (x, y, z, azimuth, elevation); kwave: device complex64
 * [n_f] (wavenumber, imaginary part = attenuation).  Replaces the per-element
 * body of the reference kernels TXfield / RXfield
 * (MATLAB/lib/simulator/SimUS_CUDARCA.cu:209-379), which the Python
 * simulator (simu_rca_ab_b200.simulator) combines with the transmit delays,
 * apodisations, pulse and impulse responses. */
int rcabf_sim_element_field(void *out, const float *r_scat, const float *r_ele, const void *kwave, float width,
                            float height, float rfocus, int baffle, float lens, float speed_of_sound,
                            int64_t n_scat, int64_t n_ele, int64_t n_f, int64_t n_sub, void *stream);

/* Transmit field of a group of n_tx transmit events that share scatterer
 * positions (n_tx <= 16):
 *   tx_out[f][s][g] = tx_factor[f] bsc[g][s]
 *                     sum_e E(f, s, e) apod[g][e] exp(i w_f delay[g][e])
 * with E the element field above (evaluated in place, not stored),
 * w_f = Re(kwave[f]) speed_of_sound, delay in seconds relative to the
 * receive start, tx_factor the conjugated pulse and transmit impulse-response
 * spectra.  tx_out: device complex64 [n_f][n_scat][n_tx]; bsc, delay, apod:
 * device float [n_tx][n_scat], [n_tx][n_ele], [n_tx][n_ele]; tx_factor:
 * device complex64 [n_f]; n_ele * n_tx <= 4096.  Replaces the reference
 * kernel TXfield and its backscatter product
 * (MATLAB/lib/simulator/SimUS_CUDARCA.cu:209-292, SimUS_CUDARCA.m:319-344). */
int rcabf_sim_tx_field(void *tx_out, const float *r_scat, const float *bsc, const float *r_ele, const void *kwave,
                       const void *tx_factor, const float *delay, const float *apod, int64_t n_tx, float width,
                       float height, float rfocus, int baffle, float lens, float speed_of_sound, int64_t n_scat,
                       int64_t n_ele, int64_t n_f, int64_t n_sub, void *stream);
/* Received spectrum of the same group:
 *   spec_out[f][e][g] = rx_factor[f] apod[g][e] sum_s E_rx(f, s, e) tx_field[f][s][g]
 * with E_rx the receive array's element field (evaluated in place) and
 * rx_factor the input-filter x receive impulse-response spectrum.
 * spec_out: device complex64 [n_f][n_ele][n_tx]; tx_field: the output of
 * rcabf_sim_tx_field; apod: device float [n_tx][n_ele].  Replaces the
 * reference kernel RXfield, the receive apodisation and the sum over
 * scatterers (SimUS_CUDARCA.cu:294-379, SimUS_CUDARCA.m:346-372). */
int rcabf_sim_rx_spectrum(void *spec_out, const void *tx_field, const float *r_scat, const float *r_ele,
                          const void *kwave, const void *rx_factor, const float *apod, int64_t n_tx, float width,
                          float height, float rfocus, int baffle, float lens, float speed_of_sound, int64_t n_scat,
                          int64_t n_ele, int64_t n_f, int64_t n_sub, void *stream);
/* Time-domain samples of the group's signals: with
 *   RF(t, e, g) = Re(ifft(conj(spec[:, e, g]), n_fast))(t)
 *              = (1 / n_fast) sum_f Re(spec[f][e][g] conj(twiddle[f t mod n_fast])) ,
 * twiddle[m] = exp(2 pi i m / n_fast) (device complex64 [n_fast]),
 * out[g][e][i] (device float [n_tx][n_ele][n_out]) holds RF(t(i)) with
 * t(i) = i for sub = 0 (the RF, zero at t >= n_fast), and for sub > 0
 * t(i) = sub (i / 2) + i mod 2: the interleave of RF(1:sub:end) and
 * RF(2:sub:end) that the reference returns as Raw.  n_f * 8 <= 49152.
 * Replaces the inverse FFT, crop / pad and sub-sampling of
 * SimUS_CUDARCA.m:374-389. */
int rcabf_sim_rf(float *out, const void *spec, const void *twiddle, int64_t n_f, int64_t n_ele, int64_t n_tx,
                 int64_t n_fast, int32_t sub, int64_t n_out, void *stream);

/* ------------------------------------------------------------------------ */
/* ULM super-localisation (downstream of the clutter filter)                 */
/* ------------------------------------------------------------------------ */
/* Maps are stacks of 2-D frames, device memory, z fastest, then x, then
 * frame: element (z, x, t) at z + nz * (x + nx * t) -- the column-major
 * layout of the reference's (Nz, Nx, Nt) ArrayFire arrays
 * (Python/superloc/superloc.py).  All calls are asynchronous on `stream`. */

/* PsfCorrMap2D (superloc.py:12-48): corr = conv(iq, conj(psf)) /
 * sqrt(conv(|iq|^2, ones)) / psf_norm per frame, ArrayFire's same-size
 * convolution (kernel element (kz/2, kx/2) on the output sample, zero
 * outside the frame).  corr, iq: complex64 [nt][nx][nz]; psf: complex64
 * [kx][kz] (column-major kz x kx); psf_norm = sqrt(sum |psf|^2) > 0;
 * kz, kx <= 33 (RCABF_ERR_UNSUPPORTED beyond). */
int rcabf_ulm_psf_corr(void *corr, const void *iq, const void *psf, float psf_norm, int64_t nz, int64_t nx,
                       int64_t nt, int32_t kz, int32_t kx, void *stream);

/* The ensemble map of SuperLocFilter (superloc.py:114-120): out(z, x, t) =
 * sqrt|sum_f ker(f) p(t + nker/2 - f)| with p(u) = map(u) conj(map(u + 1)),
 * t < nt - 1.  out: float [nt - 1][nx][nz]; map: complex64 [nt][nx][nz];
 * ker: device float [nker] (the normalised Hann window). */
int rcabf_ulm_ensemble(float *out, const void *map, const float *ker, int32_t nker, int64_t nz, int64_t nx,
                       int64_t nt, void *stream);

/* ImRegionalMax(I, 3) (superloc.py:51-53): bw = (3 x 3 dilation of map ==
 * map) per frame; bw: uint8 [nt][nx][nz]; map: float [nt][nx][nz]. */
int rcabf_ulm_regional_max(uint8_t *bw, const float *map, int64_t nz, int64_t nx, int64_t nt, void *stream);

/* Candidate pixels of SuperLocFilter (superloc.py:51-53, 122-136) on the
 * ensemble maps (float [nt][nx][nz], nt = their frame count): fit 0:
 * regional maximum (3 x 3) of corr_ens with a regional maximum of env_ens
 * within 3 x 3; fit 1: regional maximum of env_ens; z and x inside
 * [edge, n - edge).  Writes, in no particular order, the column-major
 * linear index and |value| of the fitted map (corr_ens for fit 0, env_ens
 * for fit 1) of the first `capacity` candidates to lin / val, and the total
 * candidate count to *count (device uint64). */
int rcabf_ulm_detect(int64_t *lin, float *val, uint64_t *count, const float *corr_ens, const float *env_ens,
                     int64_t nz, int64_t nx, int64_t nt, int32_t edge, int32_t fit, int64_t capacity, void *stream);

/* Sub-pixel positions of n detections (superloc.py:56-100, 140-213): for
 * each, the Hann-weighted least-squares parabola of log|map| over the
 * (2 edge + 1)^2 neighbourhood, along x and z.  The detection's (x, z,
 * frame) are read as the reference reads them, from a Fortran-flattened
 * meshgrid at the linear index L: x = (L mod nz nx) div nx, z = L mod nx,
 * frame = L div nz nx ((x, z) for square maps).  pos: device float [5][n]
 * = (x + sub-x, 0, z + sub-z, val, frame); map: float [nt][nx][nz] (the
 * fitted ensemble map); consts: device float, hann [(2e+1)^2] (z fastest),
 * roi [2e+1], the row-major inverses of the x and z moment matrices [9],
 * [9]. */
int rcabf_ulm_gauss_fit(float *pos, const int64_t *lin, const float *val, int64_t n, const float *map, int64_t nz,
                        int64_t nx, int64_t nt, int32_t edge, const float *consts, void *stream);

/* Bins of DensityMappingND / VelocityMappingND(t) (superloc.py:216-402):
 * per axis x, y, z, t the lowest bin edge, the mean bin step and the bin
 * count; positions have pos_rows values each (x, y, z, value, frame),
 * velocities vel_rows. */
typedef struct rcabf_ulm_bins {
    int32_t struct_size;   /* sizeof(rcabf_ulm_bins) */
    int32_t pos_rows;
    int32_t vel_rows;
    int32_t reserved;
    double min[4];
    double step[4];
    int64_t n[4];
} rcabf_ulm_bins;

/* Histograms of n positions (device double [n][pos_rows]): dens[z][x][y][t]
 * += 1 and, when vel is not NULL, vel[c][z][x][y][t] += vel_in[i][c]
 * (device double, zeroed by the caller).  A position's bin follows the
 * reference: (p - min) / step cast to int16 as numpy does on x86-64,
 * negatives to 0, indices past the last bin to the last bin and an index
 * equal to the bin count to 0.  use_t = 0: no time axis (t extent 1). */
int rcabf_ulm_density(double *dens, double *vel, const double *pos, int64_t n, const double *vel_in,
                      const rcabf_ulm_bins *bins, int32_t use_t, void *stream);

/* Count of device-side bound-check trips since the last call (expected 0). */
int rcabf_take_error_count(int64_t *count);

/* Number of kernel launches this library issued since the last call. */
int rcabf_take_launch_count(int64_t *count);

/* Measured FP32 FMA throughput of the current device (TFLOP/s), from a probe
 * kernel of independent FMA chains; the denominator of the beamformer's
 * FP32 roofline.  Synchronises the stream. */
int rcabf_measure_fp32_peak(double *tflops, void *stream);

/* ---------------------------------------------------------------------------
 * Casorati Gram matrix of the SVD clutter filter on the tensor cores.
 *
 * Replaces the IQf' * IQf product of SVDClutterFilter.m:23-25
 * (MATLAB/lib/clutterFilter/SVDClutterFilter.m), which the reference forms in
 * double precision before svd().  x: device complex64 [n_frame][ld], frame t's
 * n_pix pixels at x[t * ld .. t * ld + n_pix) (the beamformer's ensemble
 * layout, frame-major: the transpose of reshape(IQ, [], nT)).  G: device
 * complex128 [n_frame][n_frame], row-major, G[i][j] = sum_p conj(x[i][p])
 * x[j][p] = (C' * C)(i, j); Hermitian, written in full.
 *
 * Arithmetic: each value is cut into four signed 7-bit integer slices under a
 * power-of-two scale per (frame part, chunk of chunk_voxels pixels), the
 * slice products run on int8 tensor cores with exact int32 accumulation, and
 * the levels and chunks combine in FP64; relative to an FP64 Gram the error is
 * at most 2^-27 of each chunk's largest value per term (measured ~1e-10 of
 * max|G|), and the result is deterministic.  Chunk rows whose largest
 * magnitude is below 2^-100 count as zero.  chunk_voxels: 0 for the default
 * (16384), else a multiple of 64 up to 65536.
 * ------------------------------------------------------------------------- */
typedef struct rcabf_gram_plan {
    int32_t struct_size;      /* sizeof(rcabf_gram_plan) */
    int32_t chunk_voxels;     /* pixels per scaling chunk */
    int32_t n_chunks;
    int32_t column_block;     /* columns of the 2 n_frame x 2 n_frame real Gram per tile (MMA N) */
    int32_t n_tiles;          /* 128 x column_block tiles formed per chunk (upper triangle) */
    int32_t launches;         /* kernel launches per call */
    size_t workspace_bytes;   /* device workspace rcabf_casorati_gram needs */
    double mma_int_ops;       /* 2 x int8 multiply-adds issued to the tensor cores per call */
} rcabf_gram_plan;

int rcabf_casorati_gram_plan(int64_t n_frame, int64_t n_pix, int32_t chunk_voxels, rcabf_gram_plan *out);

/* Gram of x into G (see above); workspace: device, 256-byte aligned, at least
 * rcabf_gram_plan.workspace_bytes.  Asynchronous on `stream`.  A bounded wait
 * that gives up counts in rcabf_take_error_count. */
int rcabf_casorati_gram(void *G, const void *x, int64_t n_frame, int64_t n_pix, int64_t ld, int32_t chunk_voxels,
                        void *workspace, size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RCABF_H */
