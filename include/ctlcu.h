/*
 * ctlcu -- C ABI of the B200 cone-beam forward projector.
 *
 * A drop-in for CTL's OpenCL forward projector CTL::OCL::RayCasterProjector
 * (modules/src/projectors/raycasterprojector.h:20-58).  The C++ adapter
 * CudaRayCasterProjector (ctl_b200/adapter/) implements CTL's AbstractProjector
 * on top of these calls; the Python package ctl_b200 binds them with ctypes.
 *
 * Conventions
 *   - every call returns a ctlcu_status (0 = OK) and never throws;
 *     ctlcu_last_error() gives a readable message for the last failure on a
 *     context (thread-local to the context's lock holder, valid until the next
 *     call on that context);
 *   - a context owns one CUDA device, a CUDA stream and the volumes created on
 *     it; all calls on a context are serialised by an internal lock;
 *   - projection matrices are 3x4 row-major float64, ordered
 *     [view][module] (CTL's FullGeometry, acquisition/geometryencoder.h);
 *   - projections are float32 [view][module][row][channel] (CTL's
 *     ProjectionData / Chunk2D layout, img/projectiondata.h:19-95,
 *     img/chunk2d.tpp:477-492);
 *   - volumes are float32 on the host, x fastest, index z*X*Y + y*X + x
 *     (img/voxelvolume.tpp:310-335), centred at offset_mm.
 */
#ifndef CTLCU_H
#define CTLCU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTLCU_ABI_VERSION 2  /* 2: launch-shape fields appended to ctlcu_settings */

#if defined(__GNUC__)
#define CTLCU_API __attribute__((visibility("default")))
#else
#define CTLCU_API
#endif

typedef enum {
    CTLCU_OK = 0,
    CTLCU_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size or setting */
    CTLCU_ERR_INVALID_HANDLE = 2,   /* unknown or released volume handle */
    CTLCU_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed or memory budget exceeded */
    CTLCU_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    CTLCU_ERR_NO_DEVICE = 5,        /* device index out of range / no CUDA device */
    CTLCU_ERR_SINGULAR_GEOMETRY = 6,/* a projection matrix had a singular M; its pixels are 0 */
    CTLCU_ERR_TIMEOUT = 7,          /* reserved: no call returns it (no kernel here waits on a device-side flag) */
    CTLCU_ERR_BUSY = 8              /* admission refused (queue full) */
} ctlcu_status;

typedef enum { CTLCU_F32 = 0, CTLCU_BF16 = 1, CTLCU_F16 = 2 } ctlcu_dtype;

typedef enum {
    CTLCU_INTERP_SOFTWARE = 0, /* FP32 trilinear from the stored volume (default) */
    CTLCU_INTERP_TEXTURE = 1   /* hardware texture filter (8-bit fractional weights) */
} ctlcu_interp_mode;

typedef enum {
    CTLCU_ACCUM_FP64 = 0,  /* double accumulator, as raycasterprojector_interp.cl:48,66 */
    CTLCU_ACCUM_KAHAN = 1, /* float with compensated (Kahan) summation (default) */
    CTLCU_ACCUM_FP32 = 2   /* plain float */
} ctlcu_accum;

/*
 * Sample-loop variant.  AUTO picks CELLS for software trilinear interpolation
 * without up-sampling and GATHER otherwise.
 *   GATHER  eight scalar loads per sample from the zero-padded voxel array
 *   CELLS   one 32-byte load per sample from a derived cell array holding,
 *           per trilinear cell, the 8 coefficients of its interpolation
 *           polynomial about the cell centre (FP32, built on the device once
 *           per resident volume; 8x the voxel count x 4 bytes)
 */
typedef enum {
    CTLCU_KERNEL_AUTO = 0,
    CTLCU_KERNEL_GATHER = 1,
    CTLCU_KERNEL_CELLS = 2,
    CTLCU_KERNEL_PAIRS = 3  /* four 8-byte loads per cell from an x-pair array (mid, diff)
                               per voxel: 2x the voxel count x 4 bytes */
} ctlcu_kernel;

typedef struct ctlcu_ctx ctlcu_ctx;

typedef struct {
    uint32_t n[3];       /* voxels along x, y, z */
    float voxel_mm[3];   /* VoxelVolume::voxelSize() */
    float offset_mm[3];  /* VoxelVolume::offset() */
    int32_t dtype;       /* ctlcu_dtype used for device storage (host data is float32) */
} ctlcu_volume_desc;

/*
 * RayCasterProjector::Settings (raycasterprojector.h:27-37) plus the
 * B200 options.  ctlcu_settings_default() gives the reference defaults
 * (rays {1,1}, raySampling 0.3, volumeUpSampling 1, interpolate on) and,
 * for the B200 options, software interpolation, FP32 accumulation with
 * Kahan compensation, automatic kernel choice and launch shape.
 */
typedef struct {
    uint32_t rays_per_pixel[2]; /* sub-rays along channel (x) and row (y), 1..64 */
    float ray_sampling;         /* step / smallest voxel size, >= 1e-3 */
    uint32_t volume_upsampling; /* 0: one mean voxel, 1: as is, f>=2: f^3 replication (virtual) */
    int32_t interpolate;        /* 1 trilinear, 0 nearest voxel (forces up-sampling 1) */
    int32_t interp_mode;        /* ctlcu_interp_mode */
    int32_t accum;              /* ctlcu_accum */
    int32_t kernel;             /* ctlcu_kernel: sample-loop variant (0 = automatic) */
    /* Launch shape (no counterpart in the reference, whose OpenCL work size is
     * one work-item per pixel, raycasterprojector.cpp:339-343).  0 = the
     * autotuned value for this volume and detector (ctlcu_autotune), else the
     * default in brackets.  Results do not depend on the first three; `unroll`
     * changes only the FP32 rounding of the partial sums. */
    int32_t views_per_block;    /* views sharing a thread block: 1, 2 or 4 [2] */
    int32_t lanes_x;            /* warp patch along the channels: 4 (4x8 pixels) or 8 (8x4) [4] */
    int32_t block_rays;         /* rays (threads) per block: 128, 256 or 512 [256]; the tile is
                                   block_rays/views_per_block pixels, 16 channels wide from 128
                                   pixels up, else 8 */
    int32_t unroll;             /* cell/pair loops: samples per FP32 partial sum, 2, 4 or 8 [4] */
} ctlcu_settings;

/* One projection request of a batch: device pointers, see ctlcu_project_batch. */
typedef struct {
    uint64_t volume;       /* handle from ctlcu_volume_create */
    const double* pmats;   /* device: n_views*n_modules*12 doubles */
    float* out;            /* device: n_views*n_modules*rows*channels floats */
    uint32_t n_views, n_modules, channels, rows;
} ctlcu_request;

/* ---- context ---------------------------------------------------------------------------- */

/* Replaces OpenCLConfig::instance() + RayCasterProjector::initOpenCL
 * (ocl/openclconfig.cpp:15-38, raycasterprojector.cpp:388-422): binds one CUDA
 * device.  Fails with CTLCU_ERR_NO_DEVICE for a bad index, like
 * prepareOpenCLDeviceList (raycasterprojector.cpp:434-461). */
CTLCU_API int ctlcu_create(int device, ctlcu_ctx** out);
CTLCU_API int ctlcu_destroy(ctlcu_ctx* ctx);
CTLCU_API const char* ctlcu_last_error(const ctlcu_ctx* ctx);
CTLCU_API int ctlcu_abi_version(void);
CTLCU_API ctlcu_settings ctlcu_settings_default(void);

/* Device-memory budget for volumes (bytes, 0 = unlimited).  Creating a volume
 * beyond it fails with CTLCU_ERR_OUT_OF_MEMORY. */
CTLCU_API int ctlcu_set_memory_budget(ctlcu_ctx* ctx, uint64_t bytes);
CTLCU_API int ctlcu_memory_used(ctlcu_ctx* ctx, uint64_t* bytes);

/* The context's CUDA stream (a cudaStream_t) for callers that order their own work on it. */
CTLCU_API int ctlcu_stream(ctlcu_ctx* ctx, void** stream);

/* ---- resident volumes --------------------------------------------------------------------- */

/* Upload (data on host) or copy (data_on_device != 0) a float32 volume and
 * keep it resident in the storage dtype.  Replaces the per-call image upload
 * of raycasterprojector.cpp:239-269. */
CTLCU_API int ctlcu_volume_create(ctlcu_ctx* ctx, const ctlcu_volume_desc* desc, const float* data,
                        int data_on_device, uint64_t* handle);
CTLCU_API int ctlcu_volume_release(ctlcu_ctx* ctx, uint64_t handle);
CTLCU_API int ctlcu_volume_bytes(ctlcu_ctx* ctx, uint64_t handle, uint64_t* bytes);

/*
 * Volume cache of ctlcu_project_volume (default 0 = off: every call uploads its
 * volume and frees it, as RayCasterProjector::project does,
 * raycasterprojector.cpp:239-269).  With max_volumes > 0 the context keeps
 * resident copies (with their derived cell arrays) of the last max_volumes
 * distinct host volumes it projected; a later call whose volume has the same
 * description and the same content (a 64-bit hash of every voxel, computed on
 * the host) projects from the resident copy, without upload or cell build.
 * CTL's extensions re-project one volume many times (ArealFocalSpotExtension
 * per focal-spot sample, SpectralEffectsExtension per energy bin,
 * arealfocalspotextension.cpp:133-150, spectraleffectsextension.cpp:385-391),
 * and registration loops project one volume per pose.  Results are the same
 * with and without the cache.  The least recently used copy is evicted first;
 * setting a smaller size evicts at once.  Cached copies count against the
 * memory budget.  Device-memory volumes are never cached.
 */
CTLCU_API int ctlcu_set_volume_cache(ctlcu_ctx* ctx, uint32_t max_volumes);
/* Calls served from the cache, calls that uploaded, and copies now resident (each may be NULL). */
CTLCU_API int ctlcu_volume_cache_stats(ctlcu_ctx* ctx, uint64_t* hits, uint64_t* misses, uint32_t* resident);

/* ---- projection -------------------------------------------------------------------------- */

/*
 * RayCasterProjector::project (raycasterprojector.cpp:139-375) for a resident
 * volume: all n_views*n_modules matrices in one launch.
 * pmats and out may each be host or device memory.  With both on the device
 * the call is asynchronous on `stream` (NULL = the context's stream, which is
 * non-blocking: pass cudaStreamLegacy to order the call on the legacy default
 * stream); with either on the host the call copies on the context's stream
 * and returns when `out` is complete.
 */
CTLCU_API int ctlcu_project(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                  const double* pmats, uint32_t n_views, uint32_t n_modules, uint32_t channels,
                  uint32_t rows, float* out, void* stream);

/* One-shot form with the exact argument meaning of RayCasterProjector::project:
 * the host volume is uploaded for this call only (as the reference does), then
 * released.  Host or device pmats/out as above; returns when out is complete. */
CTLCU_API int ctlcu_project_volume(ctlcu_ctx* ctx, const ctlcu_volume_desc* desc, const float* volume,
                         const ctlcu_settings* settings, const double* pmats, uint32_t n_views,
                         uint32_t n_modules, uint32_t channels, uint32_t rows, float* out);

/*
 * Batched form: one setup launch for every request's geometry, then each
 * request's projection launch, in order on `stream`.  Requests may use
 * different volumes and detector sizes.  All pointers are device memory;
 * asynchronous on `stream` (NULL = the context's stream).  Plans
 * (ctlcu_plan_create) capture a batch once and can also run it as one
 * persistent launch.
 */
CTLCU_API int ctlcu_project_batch(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n_requests,
                        const ctlcu_settings* settings, void* stream);

/*
 * Plans: a batch prepared once (descriptors on the device, cell arrays built)
 * and captured as a CUDA graph of its setup and projection launches (in the
 * faster of two forms, below); each ctlcu_plan_launch replays it on `stream`.  The requests'
 * pmats/out pointers are fixed in the plan -- update their contents in place
 * between launches.  Plans need the cell kernel; their volumes cannot be
 * released (CTLCU_ERR_BUSY) until the plan is destroyed.
 */
typedef struct ctlcu_plan ctlcu_plan;
CTLCU_API int ctlcu_plan_create(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n_requests,
                                const ctlcu_settings* settings, ctlcu_plan** plan);
CTLCU_API int ctlcu_plan_launch(ctlcu_plan* plan, void* stream);
CTLCU_API int ctlcu_plan_destroy(ctlcu_plan* plan);

/* The two forms a plan's graph can hold.  ctlcu_plan_create captures both,
 * replays each once untimed and three times timed (writing the outputs), and
 * keeps the faster:
 *   PERSISTENT  the setup and one persistent launch over every request's work
 *               items (warp patches taken from one queue);
 *   GRIDS       the setup and one grid launch per request, the requests dealt
 *               out longest first over up to 4 parallel graph branches, so that
 *               launches overlap and fill each other's last waves.
 * Both forms give the same bits. */
typedef enum { CTLCU_PLAN_CHOOSE = -1, CTLCU_PLAN_PERSISTENT = 0, CTLCU_PLAN_GRIDS = 1 } ctlcu_plan_form;
/* The form a plan kept and the replay times (ms) measured for both at its
 * creation (0 for a plan created in a given form). */
CTLCU_API int ctlcu_plan_info(const ctlcu_plan* plan, int* form, float* ms_persistent, float* ms_grids);
/* ctlcu_plan_create in a given form (CTLCU_PLAN_PERSISTENT or CTLCU_PLAN_GRIDS),
 * without timing anything at creation; CTLCU_PLAN_CHOOSE is ctlcu_plan_create. */
CTLCU_API int ctlcu_plan_create_form(ctlcu_ctx* ctx, const ctlcu_request* requests, uint32_t n_requests,
                                     const ctlcu_settings* settings, int form, ctlcu_plan** plan);

/* ---- several devices ---------------------------------------------------------------------- */

/*
 * RayCasterProjector::Settings::deviceIDs (raycasterprojector.h:30): one
 * projection spread over several devices.  A group holds one context per
 * listed device ordinal (n_devices = 0: every device, as an empty deviceIDs
 * list means in the reference, raycasterprojector.cpp:449-454; an ordinal may
 * be listed more than once).  An unavailable ordinal fails with
 * CTLCU_ERR_NO_DEVICE, like prepareOpenCLDeviceList (:434-461).
 */
typedef struct ctlcu_group ctlcu_group;
/* Number of CUDA devices this process sees (0 when there is none). */
CTLCU_API int ctlcu_device_count(int* n);
CTLCU_API int ctlcu_group_create(const int* devices, uint32_t n_devices, ctlcu_group** out);
CTLCU_API int ctlcu_group_destroy(ctlcu_group* group);
CTLCU_API const char* ctlcu_group_last_error(const ctlcu_group* group);
CTLCU_API int ctlcu_group_size(const ctlcu_group* group, uint32_t* n_devices);
/* The context of the group's index-th device (owned by the group), for
 * per-device settings such as a memory budget. */
CTLCU_API int ctlcu_group_context(ctlcu_group* group, uint32_t index, ctlcu_ctx** ctx);

/*
 * The reference's multi-device RayCasterProjector::project
 * (raycasterprojector.cpp:187-208, :239-251, :321-357) with the argument
 * meaning of ctlcu_project_volume; volume, pmats and out are host memory.
 * min(#devices, n_views) devices take part; device i projects the contiguous
 * block of views [first[i], first[i+1]) of ctlcu_split_views with its own
 * upload of the volume, in its own host thread, into its own slice of `out`.
 * No data moves between devices.  The result equals a one-device call bit for
 * bit.  Returns when `out` is complete; the first failing device's status and
 * message (ctlcu_group_last_error) are reported.
 */
CTLCU_API int ctlcu_group_project_volume(ctlcu_group* group, const ctlcu_volume_desc* desc, const float* volume,
                                         const ctlcu_settings* settings, const double* pmats, uint32_t n_views,
                                         uint32_t n_modules, uint32_t channels, uint32_t rows, float* out);

/* The view split of ctlcu_group_project_volume (and of bench.py's ranks):
 * n_parts contiguous blocks whose sizes differ by at most one, the larger
 * ones first; part i is [first[i], first[i+1]).  first holds n_parts + 1
 * entries.  Needs no GPU. */
CTLCU_API int ctlcu_split_views(uint32_t n_views, uint32_t n_parts, uint32_t* first);

/* Wait for the context's stream; reports a deferred device-side error
 * (CTLCU_ERR_SINGULAR_GEOMETRY) raised by an earlier asynchronous call. */
CTLCU_API int ctlcu_sync(ctlcu_ctx* ctx);

/* ---- introspection used by tests and the benchmark ----------------------------------------- */

/* Exact number of volume samples the reference scheme takes for this job
 * (sum over rays of floor(tmax)+2-floor(tmin)), computed on the device. */
CTLCU_API int ctlcu_count_samples(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                        const double* pmats, uint32_t n_views, uint32_t n_modules,
                        uint32_t channels, uint32_t rows, uint64_t* samples);

/*
 * Autotuner: times the sample loops that serve these settings (cell, pair and
 * gather loops for software trilinear interpolation without up-sampling) on
 * a contiguous run of views from the middle of the job (at least `max_views`,
 * 0 = 8, lengthened until its rays fill the GPU about four times over, at most
 * the job), then, for the fastest loop, the launch shape one field at a time
 * (views per block, warp patch, rays per block, and the unroll of the cell and
 * pair loops), keeping a change that is at least 1% faster; a final shape other
 * than the default must win once more against it, timed afresh.  Launch-shape
 * fields set in `settings` stay fixed.  The result serves later calls on this volume with the same
 * detector size and module count whose kernel is CTLCU_KERNEL_AUTO (loop and
 * shape) or the tuned loop (shape); only the derived array the winner reads is
 * kept.  *kernel receives the loop; ms_out (optional) the three loop times in
 * ms (cells, pairs, gather) with the default shape.  pmats: host or device.
 */
CTLCU_API int ctlcu_autotune(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                             const double* pmats, uint32_t n_views, uint32_t n_modules, uint32_t channels,
                             uint32_t rows, uint32_t max_views, int* kernel, float* ms_out);

/* The settings a projection of this volume with this detector size and module
 * count runs with: *out = settings with the sample loop and every launch-shape
 * field resolved (autotuned where a tuning exists, else the defaults). */
CTLCU_API int ctlcu_tuned_settings(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                                   uint32_t n_modules, uint32_t channels, uint32_t rows, ctlcu_settings* out);

/* Per-(view, module) packed QR (15 doubles: Q row-major, R00 R01 R02 R11 R12 R22)
 * and per-view source position (3 doubles), computed by the device setup
 * kernel; the reference's decomposeM / determineSource
 * (raycasterprojector.cpp:527-549).  Host pointers. */
CTLCU_API int ctlcu_view_setup(ctlcu_ctx* ctx, const double* pmats, uint32_t n_views, uint32_t n_modules,
                     double* qr_out, double* src_out);

/* Number of kernels this library has launched on the context (all calls). */
CTLCU_API int ctlcu_launch_count(ctlcu_ctx* ctx, uint64_t* launches);

/* ---- post-projection operations ---------------------------------------------------------- */

/*
 * ProjectionData::transformToExtinction / transformToIntensity with one i0 per
 * view (img/projectiondata.cpp; img/singleviewdata.cpp:135-172), in place over
 * n_views x values_per_view floats: p = log(i0 / p) or p = i0 exp(-p), in FP32
 * like the reference.  i0: n_views doubles in host memory, or NULL for i0 = 1.
 * data: device memory (asynchronous on `stream`, NULL = the context's stream)
 * or host memory (returns when done).
 */
CTLCU_API int ctlcu_transform_to_extinction(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint64_t values_per_view,
                                            const double* i0, void* stream);
CTLCU_API int ctlcu_transform_to_intensity(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint64_t values_per_view,
                                           const double* i0, void* stream);

/*
 * PoissonNoiseExtension (projectors/poissonnoiseextension.cpp:35-68, :156-198) on
 * extinction data [view][module][pixel] in place: per pixel, count =
 * i0[module] exp(-p), noisy ~ Poisson(count) for count < 1e4 and
 * Normal(count, sqrt(count)) above, p = log(i0[module] / noisy).  A zero
 * count sum leaves the data unchanged, as the reference skips such views.
 * i0_per_module: n_modules photons per pixel (RadiationEncoder::photonsPerPixel),
 * host memory.  The noise of a pixel is a fixed function of (seed, view,
 * pixel): counter-based Philox4x32-10 streams instead of the reference's
 * per-view mt19937_64 (same distributions, different draws).  data: device
 * (asynchronous on `stream`) or host memory (returns when done).
 */
CTLCU_API int ctlcu_poisson_noise(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint32_t n_modules,
                                  uint32_t pixels_per_module, const float* i0_per_module, uint64_t seed,
                                  void* stream);

/* Detector saturation models (models/detectorsaturationmodels.cpp): LINEAR clamps to [a, b];
 * SPLINE is the identity between a + soft_a and b - soft_b, constant a below a - soft_a and b
 * above b + soft_b, with the reference's quadratic splines in between. */
typedef enum { CTLCU_SATURATION_LINEAR = 0, CTLCU_SATURATION_SPLINE = 1 } ctlcu_saturation_kind;
typedef struct {
    int32_t kind;          /* ctlcu_saturation_kind */
    float a, b;            /* lower and upper cap */
    float soft_a, soft_b;  /* SPLINE: half widths of the lower and upper transitions (> 0) */
} ctlcu_saturation_model;

/* Domain the saturation model acts in (AbstractDetector::SaturationModelType). */
typedef enum {
    CTLCU_SATURATION_EXTINCTION = 0,
    CTLCU_SATURATION_PHOTON_COUNT = 1,
    CTLCU_SATURATION_INTENSITY = 2
} ctlcu_saturation_domain;

/*
 * DetectorSaturationExtension (projectors/detectorsaturationextension.cpp:96-226) on extinction
 * data [view][module][pixel], in place, in FP32 as the reference computes it:
 *   extinction domain:         p = model(p)
 *   photon count / intensity:  x = s[v][k] exp(-p); x = model(x); p = log(s[v][k] / x)
 * where s[view][module] (host memory) is the incident photon count per pixel in the photon
 * count domain (SimpleCTSystem::photonsPerPixel after prepareView) and that count times the
 * mean energy of the view's spectrum in the intensity domain; NULL in the extinction domain.
 * data: device (asynchronous on `stream`) or host memory (returns when done).
 */
CTLCU_API int ctlcu_detector_saturation(ctlcu_ctx* ctx, float* data, uint32_t n_views, uint32_t n_modules,
                                        uint64_t pixels_per_module, int32_t domain,
                                        const ctlcu_saturation_model* model, const float* scale_per_view_module,
                                        void* stream);

/* ---- DEN files ---------------------------------------------------------------------------- */

/*
 * io::den::DFileFormat::save (io/den/dfileformat.tpp:148-187): writes `count`
 * row-major rows x cols matrices of elem_bytes-sized elements (1, 2, 4 or 8:
 * uchar, ushort, float, double) behind the 6-byte uint16 header.  data may be
 * device memory: it is streamed to the file through pinned staging buffers
 * (copies overlap the writes), ordered after earlier work on `stream` (NULL =
 * the context's stream).  Projections [view][module][row][channel] are
 * rows = detector rows, cols = channels, count = views x modules, as CTL's
 * DenFileIO writes them (io/den/denfileio.h:53-68).  Returns when the file is
 * complete; dimensions above 65535 are rejected, as in the reference.  ctx may
 * be NULL for host data (no GPU needed).
 */
CTLCU_API int ctlcu_den_write(ctlcu_ctx* ctx, const char* path, const void* data, uint32_t elem_bytes, uint32_t rows,
                              uint32_t cols, uint32_t count, void* stream);

/* io::den::loadHeader + getDataType (io/den/den_header.tpp:51-80, den_utils.tpp:8-24):
 * dims = {rows, cols, count}; elem_bytes from the data size. */
CTLCU_API int ctlcu_den_header(const char* path, uint32_t dims[3], uint32_t* elem_bytes);

/* DFileFormat::load (io/den/dfileformat.tpp): matrices first .. first+n-1 (n = 0: to the
 * end) into `data` (device memory, filled through pinned staging buffers, or host
 * memory) of capacity_bytes.  Returns when the data is in place.  ctx may be NULL
 * for host data. */
CTLCU_API int ctlcu_den_read(ctlcu_ctx* ctx, const char* path, void* data, uint64_t capacity_bytes, uint32_t first,
                             uint32_t n, void* stream);

/* ---- NRRD files --------------------------------------------------------------------------- */

/* BaseTypeIO<NrrdFileIO>::write(ProjectionData) (io/basetypeio.tpp:342-362,
 * io/nrrd/nrrdfileio.tpp:221-337): the header CTL writes for projections
 * (NRRD0004, float, dimension 4, sizes channels rows modules views, their labels,
 * raw little-endian, "type hint:=projection data") and the data [view][module][row][channel]
 * from device memory (streamed through pinned staging) or host memory (ctx may be NULL). */
CTLCU_API int ctlcu_nrrd_write_projections(ctlcu_ctx* ctx, const char* path, const float* data, uint32_t n_views,
                                           uint32_t n_modules, uint32_t rows, uint32_t channels, void* stream);

/* NrrdFileIO::metaInfo (io/nrrd/nrrdfileio.tpp:20-105, :352-450): the header's version,
 * dimension and sizes (fastest first), element bytes and the offset of the data.
 * Comments and key-value pairs are skipped; only raw little-endian data is accepted. */
CTLCU_API int ctlcu_nrrd_header(const char* path, uint32_t* version, uint32_t* n_dims, uint32_t sizes[4],
                                uint32_t* elem_bytes, uint64_t* data_offset);

/* NrrdFileIO::readAll: the whole data block into `data` (device memory, through pinned
 * staging, or host memory; ctx may be NULL for host memory) of capacity_bytes. */
CTLCU_API int ctlcu_nrrd_read(ctlcu_ctx* ctx, const char* path, void* data, uint64_t capacity_bytes, void* stream);

/* ---- geometry encoding ------------------------------------------------------------------- */

/* Detector of a simple CT system: CylindricalDetector(nbPixelPerModule,
 * pixelDimensions, nbDetectorModules, angulationPerModule, moduleSpacing)
 * (components/cylindricaldetector.h) or, with flat_panel = 1 and one module,
 * FlatPanelDetector (components/flatpaneldetector.h).  skew: the detector's
 * skewCoefficient (0 in CTL's stock detectors). */
typedef struct {
    uint32_t pixels[2];        /* channels, rows per module */
    double pixel_mm[2];        /* pixel width, height */
    uint32_t n_modules;
    int32_t flat_panel;
    double angulation_rad;     /* per module */
    double module_spacing_mm;
    double skew;
} ctlcu_detector_desc;

/* The stock acquisition protocols of acquisition/trajectories.h with their gantry. */
typedef enum {
    CTLCU_TRAJ_HELICAL = 0,          /* HelicalTrajectory on a TubularGantry */
    CTLCU_TRAJ_AXIAL = 1,            /* AxialScanTrajectory on a TubularGantry */
    CTLCU_TRAJ_WOBBLE = 2,           /* WobbleTrajectory on a CarmGantry */
    CTLCU_TRAJ_SHORT_SCAN = 3,       /* ShortScanTrajectory on a CarmGantry */
    CTLCU_TRAJ_CIRCLE_PLUS_LINE = 4  /* CirclePlusLineTrajectory on a CarmGantry */
} ctlcu_trajectory_kind;

typedef struct {
    int32_t kind;                 /* ctlcu_trajectory_kind */
    int32_t reserved;
    /* TubularGantry(sourceToDetectorDistance, sourceToIsoCenterDistance, -, pitchPosition, tiltAngle) */
    double sdd_mm, sid_mm, pitch_mm, tilt_rad;
    /* HelicalTrajectory(angleIncrement, pitchIncrement, startPitch, startAngle); startAngle
     * is shared with the axial and C-arm protocols */
    double angle_increment_rad, pitch_increment_mm, start_pitch_mm, start_angle_rad;
    /* CarmGantry(cArmSpan) and the C-arm protocols' sourceToIsocenter, angleSpan (a negative
     * short-scan span selects 180 deg + fan angle), wobbleAngle, wobbleFreq, lineLength,
     * fractionOfViewsForLine */
    double carm_span_mm, source_to_iso_mm, angle_span_rad, wobble_angle_rad, wobble_freq;
    double line_length_mm, line_fraction;
} ctlcu_trajectory_desc;

/*
 * GeometryEncoder::encodeFullGeometry (acquisition/geometryencoder.cpp:67-117)
 * for a simple system of the detector above on the trajectory's gantry:
 * n_views x n_modules normalised projection matrices, [view][module] 3x4
 * row-major, FP64, computed on the device in one launch.  pmats: device memory
 * (asynchronous on `stream`, NULL = the context's stream) or host memory
 * (returns when the matrices are written).
 */
CTLCU_API int ctlcu_encode_geometry(ctlcu_ctx* ctx, const ctlcu_detector_desc* detector,
                                    const ctlcu_trajectory_desc* trajectory, uint32_t n_views, double* pmats,
                                    void* stream);

/* The same for n_shifts source displacements at once: each shift (x, y, z in mm,
 * in the source's own frame, host memory) is added to the prepared gantry's source
 * displacement as a GantryDisplacementParam increment does
 * (acquisition/preparesteps.cpp:202-210, components/abstractgantry.h:159-164);
 * ArealFocalSpotExtension uses this for its focal-spot samples
 * (projectors/arealfocalspotextension.cpp:108-127).  pmats: [shift][view][module]. */
CTLCU_API int ctlcu_encode_geometry_shifted(ctlcu_ctx* ctx, const ctlcu_detector_desc* detector,
                                            const ctlcu_trajectory_desc* trajectory, uint32_t n_views,
                                            const double* source_shifts_mm, uint32_t n_shifts, double* pmats,
                                            void* stream);

/* ArealFocalSpotExtension's averaging (projectors/arealfocalspotextension.cpp:127-160):
 * out[i] = -log(mean_s exp(-in[s][i])) over n_samples projections [sample][values]
 * (intensity domain), or mean_s in[s][i] with low_extinction != 0.  Device memory,
 * asynchronous on `stream` (NULL = the context's stream). */
CTLCU_API int ctlcu_average_samples(ctlcu_ctx* ctx, const float* in, uint32_t n_samples, uint64_t values_per_sample,
                                    float* out, int low_extinction, void* stream);

/* DynamicProjectorExtension over a LinearDynamicVolume (projectors/dynamicprojectorextension.cpp:37-60,
 * img/lineardynamicvolume.cpp:194-198): the reference re-projects each view with the voxels set to
 * slope * float(t_view) + offset.  The projection is linear in the voxel values, so from the
 * projections of the slope and the offset volumes over all views:
 * out[view] = float(times[view]) * slope_proj[view] + offset_proj[view].
 * times: n_views seconds, host memory; projections device memory, asynchronous on `stream`. */
CTLCU_API int ctlcu_combine_linear(ctlcu_ctx* ctx, const float* slope_proj, const float* offset_proj,
                                   const double* times, uint32_t n_views, uint64_t values_per_view, float* out,
                                   void* stream);

/* SpectralEffectsExtension, linear case (projectors/spectraleffectsextension.cpp:215-278,
 * :333-353): from the projections of the materials' density volumes
 * (material_projs [material][view][...], device), per pixel of view v
 *   out = log(total_intensity[v] / sum_b intensities[b][v] exp(-sum_m mu_per_mm[b][m] proj_m) response[b])
 * in FP32 as the reference computes it; bins whose intensities sum to zero are skipped.
 * mu_per_mm [bin][material] (mass attenuation x 0.1, cm -> mm), intensities [bin][view],
 * response [bin] (NULL: no detector response model) and total_intensity [view] are
 * host memory, from CTL's spectral models (RadiationEncoder, attenuation models).
 * out: device; returns when done. */
CTLCU_API int ctlcu_spectral_combine(ctlcu_ctx* ctx, const float* material_projs, uint32_t n_materials,
                                     uint32_t n_views, uint64_t values_per_view, const float* mu_per_mm,
                                     const double* intensities, const float* response, uint32_t n_bins,
                                     const double* total_intensity, float* out, void* stream);

/* SpectralEffectsExtension around a non-linear nested chain, projector | PoissonNoiseExtension
 * (projectors/spectraleffectsextension.cpp:285-314, :368-391).  The reference projects, per energy
 * bin, each material's attenuation volume mu_m(E_b) * density_m through the nested chain, so each
 * (bin, material) projection gets its own noise with the bin's photon count.  The projector is
 * linear, so that projection is mu_per_mm[b][m] * material_projs[m]: one projection per material
 * replaces bins x materials, and only the noise runs per (bin, material).  Per pixel of view v and
 * module k:
 *   e'_bm = log(i0[b][k] / n_bm),  n_bm ~ Poisson(i0[b][k] exp(-mu_per_mm[b][m] proj_m))
 *   out   = log(total_intensity[v] / sum_b intensities[b][v] exp(-sum_m e'_bm) response[b])
 * The draw for (b, m) is ctlcu_poisson_noise's with seed + c, c counting the (bin, material)
 * projections of the bins not skipped in the reference's loop order (a fixed-seed noise
 * extension's successive calls).  Bins whose intensities sum to zero are skipped; a bin whose i0
 * sums to zero passes without noise.  i0_per_bin_module [bin][module] and the other spectral
 * inputs as for ctlcu_spectral_combine, host memory; material_projs [material][view][module]
 * [pixel] and out device memory.  Returns when done. */
CTLCU_API int ctlcu_spectral_combine_noisy(ctlcu_ctx* ctx, const float* material_projs, uint32_t n_materials,
                                           uint32_t n_views, uint32_t n_modules, uint64_t pixels_per_module,
                                           const float* mu_per_mm, const double* intensities,
                                           const float* response, uint32_t n_bins,
                                           const double* total_intensity, const float* i0_per_bin_module,
                                           uint64_t seed, float* out, void* stream);

/*
 * No counterpart in the reference.  ctlcu_project for callers that cannot
 * allocate device memory while they run: a real-time loop that reserved all
 * of its memory up front, or a host whose allocator must not be entered
 * (an allocation can synchronise the device or fail when memory is full).
 * This call makes no device allocation.  The per-(view, module) ray geometry
 * goes into one fixed scratch array in the library's static device memory:
 * CTLCU_NOALLOC_MAX_VIEW_MODULES entries of 104 bytes (416 KiB), held on every
 * device that loads the library until the process exits.  A call with more
 * than that many view-modules (n_views * n_modules) fails with
 * CTLCU_ERR_INVALID_ARGUMENT; split it.
 *  - pmats and out must be device memory (host buffers would need staging
 *    memory); asynchronous on `stream` as ctlcu_project; singular matrices
 *    are reported by ctlcu_sync.
 *  - Every derived array the settings read (the cell or pair array, the
 *    mean-voxel volume, a texture) must exist already, built by an earlier
 *    ctlcu_project or ctlcu_autotune of this volume with these settings;
 *    otherwise CTLCU_ERR_INVALID_ARGUMENT names the missing one.
 *  - The first call on a device looks up the scratch array's address there
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *    The address is kept for the life of the process: after cudaDeviceReset
 *    (or any teardown of the device's primary context) this call must not be
 *    used on that device again.
 *  - Every call on a device shares the one scratch array: calls whose work
 *    overlaps on the GPU (on different streams or contexts) race on it, so
 *    serialise them (one stream, or events between them).
 */
#define CTLCU_NOALLOC_MAX_VIEW_MODULES 4096
CTLCU_API int ctlcu_project_noalloc(ctlcu_ctx* ctx, uint64_t volume, const ctlcu_settings* settings,
                                    const double* pmats, uint32_t n_views, uint32_t n_modules,
                                    uint32_t channels, uint32_t rows, float* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
