/*
 * fdk.h -- C ABI of the B200-native FDK reconstructor (libfdk_b200.so).
 *
 * The entry points replace the reference's plugin boundaries (peng-ac/fdk):
 *   - the FDK geometry core   (common/type.h  Parameter, filter(), CalculateCosTable,
 *                              CalculateProjMat)
 *   - the CPU filter plugin   (Filterlib/FilterLib.h  FilterEngine)
 *   - the GPU filter plugin   (FilterlibCufft/cudaFftFilter.cuh  FilterRow_Real32,
 *                              CorrectImage_Real32)
 *   - the backprojection      (cudaBP/backprojection.cuh  BackProjectionFDK)
 *   - the RTK-style drop-in   (cudaBP/rtkCudaFDKBackProjectionImageFilter.cu
 *                              CUDA_reconstruct_conebeam)
 * Each declaration cites the reference interface it replaces.
 *
 * Conventions
 *   - Plain pointers and sizes only; no C++ or torch types cross this ABI.
 *   - Every function returns an int status: FDK_OK (0) or a negative FDK_ERR_*.
 *     Nothing throws across the ABI.  fdk_last_error() returns a thread-local
 *     message for the last failing call on the calling thread.
 *   - "host" pointers are CPU memory (pageable or pinned); "dev" pointers are
 *     device memory on the handle's device.
 *   - Handles are not thread-safe: one host thread drives one handle, as the
 *     reference drives one BackProjectionFDK per GPU from one BpThread
 *     (cuFDK/mpiFDK.cpp:205-317).
 *   - stream arguments are cudaStream_t passed as void* (NULL = legacy default
 *     stream).
 */
#ifndef FDK_B200_FDK_H
#define FDK_B200_FDK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDK_ABI_VERSION 1

/* ---- status codes --------------------------------------------------------- */
#define FDK_OK 0
#define FDK_ERR_INVALID_ARG (-1)   /* bad size, pointer, layout or state */
#define FDK_ERR_CUDA (-2)          /* a CUDA runtime call failed */
#define FDK_ERR_OUT_OF_MEMORY (-3) /* device or pinned-host allocation failed */
#define FDK_ERR_TIMEOUT (-4)       /* a bounded wait (host or device) ran out */
#define FDK_ERR_UNSUPPORTED (-5)   /* valid request this build does not implement */
#define FDK_ERR_NO_DEVICE (-6)     /* no CUDA device visible */
#define FDK_ERR_DEVICE_CHECK (-7)  /* a kernel reported an internal check failure */
#define FDK_ERR_IO (-8)            /* a file could not be opened, read or written, or has the wrong size */

const char *fdk_last_error(void);
int fdk_abi_version(void);
/* Number of visible CUDA devices (0 without a GPU; not an error). */
int fdk_device_count(int *count);

/* ---- geometry: Parameter (common/type.h:4627-4895) ------------------------ */
/* Filter windows, in the order of s_FILTER_TYPE (common/type.h:4619-4626). */
#define FDK_FILTER_NONE 0
#define FDK_FILTER_RAM_LAK 1
#define FDK_FILTER_SHEPP_LOGAN 2
#define FDK_FILTER_COSINE 3
#define FDK_FILTER_HAMMING 4
#define FDK_FILTER_HANN 5

typedef struct fdk_geometry {
    int64_t nx, ny, nz;          /* volume size in voxels */
    double dx, dy, dz;           /* voxel pitch, mm */
    int64_t nu, nv;              /* detector columns, rows */
    double du, dv;               /* detector pitch, mm */
    double offset_nu, offset_nv; /* detector offsets in pixels (cos table only, as in the reference) */
    double sid;                  /* source-to-detector distance, mm (reference "SID") */
    double sod;                  /* source-to-axis distance, mm (reference "SOD") */
    int64_t direction;           /* rotation direction, +1 or -1 */
    double scan_angle;           /* degrees covered by n_proj views */
    int64_t n_proj;              /* number of views */
    double volume_position_angle; /* radians added to every view angle (reference volume_postion_angle) */
    int32_t filter_type;         /* FDK_FILTER_* */
    int32_t reserved;
} fdk_geometry;

/* Parameter::Parameter() defaults (common/type.h:4628-4662). */
void fdk_geometry_default(fdk_geometry *g);
/* nextpow2 (common/type.h:4418-4425): filter length W for nu columns (doubles exact powers of two). */
int64_t fdk_filter_length(int64_t nu);
/* filter(strType, len, d) (common/type.h:4427-4475): W = fdk_filter_length(len) FP64 taps of the
 * frequency response, written to out (capacity out_len >= W). */
int fdk_filter_design(int32_t filter_type, int64_t len, int32_t d, double *out, int64_t out_len);
/* AngularAndrampFactor (common/type.h:4736). */
int fdk_angular_ramp_factor(const fdk_geometry *g, double *out);
/* cos_sigma table, nv rows of nu (CalculateCosTable, common/type.h:4756-4783):
 * SID/sqrt(u^2+v^2+SID^2) * SOD^2 * AngularAndrampFactor, FP32 storage. */
int fdk_cos_table(const fdk_geometry *g, float *out);
/* csc_sigma table: 1 / cos_sigma of the stored FP32 cos_sigma, in FP64, stored FP32
 * (common/type.h:4760, 4784). */
int fdk_csc_table(const fdk_geometry *g, float *out);
/* Per-view angles in radians: direction*deg/180*pi + volume_position_angle, deg = i*scan_angle/n_proj
 * (common/type.h:4729, 4824). */
int fdk_view_angles(const fdk_geometry *g, double *out);
/* 3x4 projection matrices, 12 per view, row major (CalculateProjMat, common/type.h:4898-4944;
 * vec_rot_mat_ijk3x4 4821-4831).  Computed in FP64; out_f64 and/or out_f32 may be NULL. */
int fdk_projection_matrices(const fdk_geometry *g, double *out_f64, float *out_f32);

/* ---- filter: FilterEngine (Filterlib/FilterLib.h:148-203) ----------------- */
/* Output element type of the device filter. */
#define FDK_DTYPE_F32 0
#define FDK_DTYPE_F16 1
/* Output layout of the device filter.
 *   ROWS       nv rows of nu (the input layout; FilterEngine transpose=false)
 *   TRANSPOSED nu rows of nv  (FilterEngine transpose=true; the BackProjectionFDK input)
 *   MIRROR     nu rows of nv mirror pairs: element (u, v) holds the filtered values of detector
 *              rows v and nv-1-v.  This is the backprojection's internal staging layout. */
#define FDK_LAYOUT_ROWS 0
#define FDK_LAYOUT_TRANSPOSED 1
#define FDK_LAYOUT_MIRROR 2

typedef struct fdk_filter fdk_filter;
/* FilterEngine(cos_image_table, fft_kernel_real_f32) (FilterLib.h:152-164).
 * cos_table: host, nv rows of nu (NULL = no cosine weighting).  H: host, W taps.
 * pad_edge: samples averaged for the constant edge pad -- 4 as the IPP plugin
 * (FilterLib.h:38,44), 3 as the cuFFT plugin (cudaFftFilter.cu:25,29).
 * W must be a power of two, nu <= W <= 4096. */
int fdk_filter_create(fdk_filter **out, const float *cos_table, const float *H, int64_t nu, int64_t nv,
                      int64_t W, int32_t pad_edge, int32_t device);
/* FilterEngine::Filtering(src, dst, transpose) (FilterLib.h:167-196): one view, host buffers.
 * As in the reference, src is cosine-weighted in place.  dst is nv x nu, or nu x nv if transpose. */
int fdk_filter_filtering(fdk_filter *h, float *src_host, float *dst_host, int32_t transpose);
/* Device batch: n_views views (nv x nu each, contiguous) -> dst in `layout` and `out_dtype`,
 * every output sample multiplied by out_scale (FP16 range control; 1 = none).  Cosine
 * weighting is applied on the fly (src is not modified).  Asynchronous on stream. */
int fdk_filter_run_device(fdk_filter *h, const float *src_dev, void *dst_dev, int64_t n_views,
                          int32_t layout, int32_t out_dtype, float out_scale, void *stream);
int fdk_filter_destroy(fdk_filter *h);

/* The same filter as a GEMM on the tensor cores (no reference counterpart: a Toeplitz
 * row-GEMM, 16-bit operands, FP32 accumulation).  Per row, y = M (in_scale * cos * p) with M
 * the nu x nu matrix of the fused filter (edge-mean pads, circular kernel IDFT(H), crop; built in
 * FP64, stored FP16 or BF16 when bf16 != 0).  split != 0 keeps the low parts of both operands
 * (x_hi M_hi + x_lo M_hi + x_hi M_lo, three times the FLOPs, close to FP32 accuracy).  nu must be
 * a multiple of 256, nv of 128, and the device an sm_100 GPU (FDK_ERR_UNSUPPORTED otherwise). */
typedef struct fdk_toeplitz fdk_toeplitz;
int fdk_toeplitz_create(fdk_toeplitz **out, const float *cos_table, const double *H, int64_t nu, int64_t nv,
                        int64_t W, int32_t pad_edge, int32_t bf16, int32_t split, float in_scale, int32_t device);
/* n_views raw FP32 views (nv x nu each, device) -> FP16 output * out_scale, ROWS or MIRROR
 * layout, asynchronous on stream. */
int fdk_toeplitz_run_device(fdk_toeplitz *h, const float *dev_src, void *dev_dst, int64_t n_views, int32_t layout,
                            float out_scale, void *stream);
/* After a sync: FDK_ERR_DEVICE_CHECK if a pipeline wait timed out or an output left the FP16 range. */
int fdk_toeplitz_check(fdk_toeplitz *h);
/* The FP64 filter matrix M (nu x nu, row-major, out[u * nu + c]) of filter response H (W taps). */
int fdk_toeplitz_matrix(const double *H, int64_t W, int64_t nu, int32_t pad_edge, double *out);
int fdk_toeplitz_destroy(fdk_toeplitz *h);

/* FilterlibCufft plugin (FilterlibCufft/cudaFftFilter.cuh:6-8, cudaFftFilter.cu:283-392).
 * DataRef<float> (FilterlibCufft/cudaBackProjection.cuh:121-230) as a plain struct: device data,
 * width (fast axis), height, depth, pitch in elements.
 * fdk_correct_image_real32: dst = src * table per view (kernelCorrect, cudaFftFilter.cu:270-281).
 * fdk_filter_row_real32: ramp filter of every row of every view with the W-tap response in
 * `filter` (pad with the mean of 3 edge samples, cudaFftFilter.cu:14-61).  Synchronous, as the
 * reference. */
typedef struct fdk_dataref {
    float *data;
    int32_t width, height, depth, pitch;
} fdk_dataref;
int fdk_correct_image_real32(const fdk_dataref *src, const fdk_dataref *table, fdk_dataref *dst);
int fdk_filter_row_real32(const fdk_dataref *src, fdk_dataref *dst, const fdk_dataref *filter);
/* No counterpart in the reference.  fdk_filter_row_real32 without any device allocation, for
 * callers that cannot allocate device memory when they filter (they reserve the device budget up
 * front, or cannot afford cudaMalloc/cudaFree, which may synchronise the device, in their
 * processing loop).  The FFT tables live in a 32 KiB file-scope device array of the library that
 * every GPU using the library holds until the process exits; filter->width (W) must be at most
 * 4096, larger W is rejected with FDK_ERR_INVALID_ARG.  All calls share the array and each call
 * rewrites the entries it uses; calls that overlap on one GPU (from several host threads) race
 * and must be serialised by the caller.  Each call looks up the array's address on the current
 * device; the first call on a device also loads the library's device code there, so make that
 * first call before starting any stream capture.  Synchronous, like the original: the kernels run
 * on the legacy default stream and the call returns once that stream has finished them. */
int fdk_filter_row_real32_noalloc(const fdk_dataref *src, fdk_dataref *dst, const fdk_dataref *filter);

/* ---- backprojection: BackProjectionFDK (cudaBP/backprojection.cuh:246-271) -- */
/* Arithmetic of the backprojection kernel.
 *   FP32_EXACT  the reference kernel's arithmetic (cudaFdkBP, backprojectionFDK.cu:50-129:
 *               FP32, mad.rz.ftz blends), bit-identical results; views read through L1.
 *   FP32        FP32 views staged in shared memory, FP32 accumulation (plain FP32 fast path).
 *   MIXED       FP16 views staged in shared memory, FP32 compensated accumulation. */
#define FDK_BP_FP32_EXACT 0
#define FDK_BP_FP32 1
#define FDK_BP_MIXED 2

/* geo::BoxT<size_t> (cudaBP/backprojection.cuh:66-116): origin and extent in voxels. */
typedef struct fdk_box {
    uint64_t x, y, z, width, height, depth;
} fdk_box;

typedef struct fdk_bp fdk_bp;
/* BackProjectionFDK(projW, projH, projCount, nx, ny, nz, subTop, subBottom)
 * (backprojectionFDK.cu:161-227).  proj_width/proj_height: the transposed view (width = nv,
 * height = nu, cuFDK/mpiFDK.cpp:196).  proj_count: views per BP() call (<= 32 as MAX_PROJ).
 * sub_bottom->depth > 0 selects the mirror-symmetric slab pair; then
 * sub_top->z + sub_bottom->z + sub_bottom->depth - 1 == nz - 1 (:171-173).
 * The volume is zeroed on creation. */
int fdk_bp_create(fdk_bp **out, int32_t proj_width, int32_t proj_height, int32_t proj_count,
                  int32_t nx, int32_t ny, int32_t nz, const fdk_box *sub_top,
                  const fdk_box *sub_bottom, int32_t precision, int32_t device);
/* BP(TRANSPOSE, pProjData, width, height, pProjMat, nProj) (backprojectionFDK.cu:229-276).
 * host_proj: n_proj views, host memory; copied before return, so the caller may reuse it.
 * transpose = 1: views are height (= nu) rows of width (= nv) values, the production layout.
 * transpose = 0: views are nv rows of nu.  proj_mat: 12 floats per view (host). */
int fdk_bp_bp(fdk_bp *h, int32_t transpose, const float *host_proj, int32_t width, int32_t height,
              const float *proj_mat, int32_t n_proj);
/* Device-resident variant: views already on the device in FDK_LAYOUT_TRANSPOSED (f32) or
 * FDK_LAYOUT_MIRROR (f32 or f16 per the handle's precision), n_proj <= 128.  Asynchronous on
 * stream; dev_proj must stay valid until the stream passes this call. */
int fdk_bp_bp_device(fdk_bp *h, const void *dev_proj, int32_t layout, const float *proj_mat,
                     int32_t n_proj, void *stream);
/* GetVolumeData(pVol, size) (backprojectionFDK.cu:278-362): writes the sub-volume as
 * [zs][y][x] (x fastest), zs = top slab then bottom slab, each ascending.  Synchronous. */
int fdk_bp_get_volume(fdk_bp *h, float *host_vol, int64_t size);
/* Device pointer of the internal volume ([x][y][zs], zs fastest) and its size in floats. */
int fdk_bp_volume_device(fdk_bp *h, float **dev_vol, int64_t *count);
/* No counterpart in the reference (accuracy checks of volumes too large to read back whole).
 * Values of n listed voxels, host_xyz = n triples (x, y, z) of whole-volume indices, into
 * host_out (n floats); voxels outside the handle's boxes read NaN.  Waits (bounded) for the
 * handle's launches first; MIXED folds its compensation term. */
int fdk_bp_sample(fdk_bp *h, const int32_t *host_xyz, int64_t n, float *host_out);
/* nBpCount, fKernelTime (cudaBP/backprojection.cuh:130, 265): views backprojected and the summed
 * kernel time in ms (events on the handle's stream). */
int fdk_bp_stats(fdk_bp *h, int64_t *bp_count, double *kernel_ms);
/* Zero the volume (start a new reconstruction with the same handle). */
int fdk_bp_reset(fdk_bp *h);
int fdk_bp_destroy(fdk_bp *h);

/* ---- RTK drop-in: CUDA_reconstruct_conebeam
 *      (cudaBP/rtkCudaFDKBackProjectionImageFilter.cu:200-330) ---------------- */
/* proj_size = {width (u), height (v), n_proj <= 32}, vol_size = {nx, ny, nz}.
 * matrices: host, 12 floats per view (index -> (u*w, v*w, w)).  dev_vol_in/dev_vol_out: device,
 * x fastest; dev_vol_out = dev_vol_in + sum_p bilinear(proj_p; u, v) / w^2.  proj: HOST views,
 * u fastest (the reference copies it with cudaMemcpyHostToDevice, :256).  Synchronous. */
int fdk_rtk_reconstruct_conebeam(const int32_t proj_size[3], const int32_t vol_size[3],
                                 const float *matrices, const float *dev_vol_in, float *dev_vol_out,
                                 const float *proj);
/* The same backprojection on views already in device memory (no reference counterpart): host_mats
 * 12 floats per view, up to 128 views, dev_proj n frames of height x width (u fastest).
 * Asynchronous on stream; vol_out may equal vol_in. */
int fdk_rtk_backproject_device(const int32_t proj_size[3], const int32_t vol_size[3], const float *host_mats,
                               const float *dev_vol_in, float *dev_vol_out, const float *dev_proj, void *stream);
/* Wait for stream and report (then clear) a device-side failure of the staged RTK kernel: its
 * bounded pipeline waits ran out (FDK_ERR_DEVICE_CHECK).  fdk_rtk_reconstruct_conebeam checks
 * this itself; callers of fdk_rtk_backproject_device call it after their launches. */
int fdk_rtk_sync(void *stream);

/* ---- end-to-end streaming FDK (single-GPU analogue of cuFDK's
 *      FilterThread -> BpThread handoff, cuFDK/mpiFDK.cpp:58-317) ------------- */
typedef struct fdk_recon fdk_recon;
/* A reconstructor for geometry g: cosine weight + ramp filter + backprojection of the whole
 * volume (mirror slab pair, as DivVolume with one rank, cuFDK/mpiFDK.h:116-149).
 * batch: views per backprojection batch (<= 512; <= 32 for FDK_BP_FP32_EXACT), independent of
 * how many views each push carries.  Two batches of filtered views stay on the device.
 * precision: FDK_BP_*. */
int fdk_recon_create(fdk_recon **out, const fdk_geometry *g, int32_t precision, int32_t batch,
                     int32_t device);
/* The same for one mirror-symmetric slab pair of the volume (one rank of DivVolume,
 * cuFDK/mpiFDK.h:116-149): top slab z in [top_z, top_z + depth), bottom slab
 * z in [nz - top_z - depth, nz - top_z).  fdk_recon_get_volume then returns the pair as
 * [zs][y][x] with zs = top slab then bottom slab, ascending. */
int fdk_recon_create_slab(fdk_recon **out, const fdk_geometry *g, int64_t top_z, int64_t depth,
                          int32_t precision, int32_t batch, int32_t device);
/* The reconstructor's compute stream (cudaStream_t as void*), for event timing by the caller. */
int fdk_recon_stream(fdk_recon *h, void **stream);
/* Push n raw views (host, nv x nu each, index first..first+n-1; pinned memory overlaps best).
 * Views may come in any order; a batch of the staged precisions holds whatever views arrived
 * (FP32_EXACT batches hold consecutive views).
 * The copy to the device runs on a side stream; filtering and backprojection follow on the
 * compute stream.  Returns once the host buffer may be reused. */
int fdk_recon_push(fdk_recon *h, const float *host_views, int64_t first, int64_t n);
/* Push n raw views already in device memory (nv x nu each). */
int fdk_recon_push_device(fdk_recon *h, const float *dev_views, int64_t first, int64_t n);
/* No counterpart in the reference.  Push n raw views whose indices are views[0..n) (any order,
 * each in 0..n_proj-1), stored one after another in host_views (pinned memory overlaps best) or
 * dev_views: one copy and one filter launch for views the caller reads out of order, e.g. a few
 * consecutive views from each quarter of the scan, so that the quarter-turn kernel
 * (fdk_recon_bp_kernel) finds whole orbits in every batch.  Returns as fdk_recon_push. */
int fdk_recon_push_views(fdk_recon *h, const float *host_views, const int64_t *views, int64_t n);
int fdk_recon_push_device_views(fdk_recon *h, const float *dev_views, const int64_t *views, int64_t n);
/* Push views first..first+n-1 from a projection folder (files as fdk_proj_path, view v in file
 * v * step + start).  Files are read by `threads` host threads (<= 0: up to 8) into two pinned
 * staging buffers of one batch each, so reading batch k+1 overlaps the copy and the kernels of
 * batch k.  Every file's size is checked before any is read (FDK_ERR_IO names the first bad one). */
int fdk_recon_push_folder(fdk_recon *h, const char *folder, int64_t first, int64_t n, int32_t step,
                          int32_t start, int32_t threads);
/* Pushed views are filtered at once and backprojected a full batch at a time; a full batch runs
 * when the next batch starts (views that do not continue the waiting ones close them first).
 * fdk_recon_flush launches the backprojection of everything waiting now (asynchronous; two
 * waiting batches run z band by z band); fdk_recon_sync and fdk_recon_get_volume flush
 * implicitly. */
int fdk_recon_flush(fdk_recon *h);
/* The row filter this reconstructor runs: 0 the FFT filter (fdk_filter_*), 1 the split-FP16
 * tensor-core GEMM (fdk_toeplitz_*, MIXED precision when nu % 256 == 0 and nv % 128 == 0 on an
 * sm_100 GPU, unless the environment sets FDK_FILTER=fft). */
int fdk_recon_filter_kind(fdk_recon *h, int32_t *kind);
/* The backprojection this reconstructor runs: 0 the reference arithmetic (FP32_EXACT), 1 the
 * staged kernel, 2 the staged kernel plus the quarter-turn kernel: views whose partners
 * v + N/4, v + N/2, v + 3N/4 (mod N) are in the same batch are backprojected four at a time
 * with one address computation (a circular scan of N % 4 == 0 views about a square, centred
 * grid).  FP32 uses it by default; MIXED only when the environment sets FDK_BP_SYM=1 (its
 * staged kernel measured faster); FDK_BP_SYM=0 turns it off.  No counterpart in the reference. */
int fdk_recon_bp_kernel(fdk_recon *h, int32_t *kind);
/* Wait (bounded by timeout_ms; <= 0 means 10 minutes) until every pushed view is backprojected. */
int fdk_recon_sync(fdk_recon *h, int64_t timeout_ms);
/* Volume [z][y][x], x fastest, nz*ny*nx floats (host; the slab pair for a slab reconstructor).
 * Implies fdk_recon_sync.  Large volumes are backprojected in z bands; each band is copied out
 * as soon as the last batch has finished it, so most of the copy overlaps that batch. */
int fdk_recon_get_volume(fdk_recon *h, float *host_vol, int64_t size);
/* fdk_bp_sample on the reconstructor's volume, after fdk_recon_sync (no counterpart in the
 * reference): n voxels (x, y, z) of the whole volume; voxels outside the slab pair read NaN. */
int fdk_recon_sample(fdk_recon *h, const int32_t *host_xyz, int64_t n, float *host_out);
/* Timing: total BP kernel ms, total filter kernel ms, views done. */
int fdk_recon_stats(fdk_recon *h, double *bp_ms, double *filter_ms, int64_t *views);
/* Kernel launches (filter and backprojection) since creation or the last reset. */
int fdk_recon_launch_count(fdk_recon *h, int64_t *count);
int fdk_recon_reset(fdk_recon *h);
int fdk_recon_destroy(fdk_recon *h);

/* ---- on-disk formats (common/type.h, cuFDK/mpiFDK.cpp) ----------------------- */
/* Path of view `view`'s raw file: folder + "img%04d.raw" % (view * step + start)
 * (Parameter::GetProjPath, common/type.h:4847-4851; folder carries its trailing '/'). */
int fdk_proj_path(const char *folder, int64_t view, int32_t step, int32_t start, char *out, int32_t capacity);
/* Views first..first+count-1 from a projection folder into host_views (count x nv x nu FP32, u
 * fastest), `threads` readers (<= 0: up to 8).  As LoadProjectionImageFolder (common/type.h:1797-1828)
 * every file must hold exactly nu * nv FP32 values, checked before any is read. */
int fdk_load_proj_folder(const char *folder, int32_t nu, int32_t nv, int64_t first, int64_t count, int32_t step,
                         int32_t start, float *host_views, int32_t threads);
/* Views to folder + img%04d.raw % ((first + i) * step), creating the folder (SaveToFolder,
 * common/type.h:3848-3861). */
int fdk_save_proj_folder(const char *folder, const float *host_views, int32_t nu, int32_t nv, int64_t first,
                         int64_t count, int32_t step, int32_t threads);
/* ".vol": int32 nx, ny, nz, then nx*ny*nz FP32 voxels [z][y][x] (VolumeT::Save/Load,
 * common/type.h:3256-3313).  fdk_load_volume with host_vol NULL only reads the header. */
int fdk_save_volume(const char *path, const float *host_vol, int32_t nx, int32_t ny, int32_t nz);
int fdk_load_volume(const char *path, float *host_vol, int64_t capacity, int32_t *nx, int32_t *ny, int32_t *nz);
/* Slices z0..z0+depth-1 of a [z][y][x] block (host_vol starts at slice z0), one raw FP32 file of
 * nx*ny per slice named folder + "%06d.raw" % z (the slice writer of cuFDK/mpiFDK.cpp:548-576). */
int fdk_save_volume_slices(const char *folder, const float *host_vol, int32_t nx, int32_t ny, int32_t z0,
                           int32_t depth, int32_t threads);

/* ---- synthetic data: analytic ellipsoid projections on the device ---------- */
/* ell: host, n_ell records of 16 doubles {cx, cy, cz, a, b, c, R00..R22, rho} in the world frame
 * of CalculateProjMat (X = (x-(nx-1)/2)dx, Y = -(y-(ny-1)/2)dy, Z = -(z-(nz-1)/2)dz, mm;
 * world = R * local).  Writes n views (first..first+n-1) of exact line integrals, nv x nu each,
 * to dev_out (f32).  Asynchronous on stream. */
int fdk_phantom_project(const fdk_geometry *g, const double *ell, int32_t n_ell, int64_t first,
                        int64_t n, float *dev_out, void *stream);

/* ---- ray-marching forward projector: kernel_forwardProject
 *      (genProj/cudaForwardProjection.cu:174-254, Text3DLinear genProj/cudaIterType.cuh:232-276) */
/* dev_vol: device volume [z][y][x] (x fastest) of g's size.  Writes views first..first+n-1, nv x nu
 * each, to dev_out: per detector pixel, trilinear samples every min(dx, dy, dz) mm along the ray
 * inside the voxel-centre box, times the step.  Asynchronous on stream (returns after queueing). */
int fdk_forward_project(const fdk_geometry *g, const float *dev_vol, int64_t first, int64_t n, float *dev_out,
                        void *stream);

/* ---- learned residual row filter and its training kernels (no reference counterpart) -------
 * Network per detector row x (length <= 256): a1 = relu(W1*(s x)+b1) (1->32 channels, kernel 9,
 * zero 'same' padding), a2 = relu(W2*a1+b2) (32->32), o = W3*a2+b3 (32->1), y = x + o/s; s scales
 * rows to line-integral units.  Parameters FP32 in the order W1[32][9], b1[32], W2[32][32][9], b2[32],
 * W3[32][9], b3 (fdk_nn_param_count() floats); activations BF16 in shared memory. */
int fdk_nn_param_count(void);
/* y = x + net(x) for `rows` rows of `len` samples (device, row-major). */
int fdk_nn_forward(const float *params, const float *x, float *y, int64_t rows, int32_t len, float scale,
                   void *stream);
/* Parameter gradient dparams (overwritten) of sum(dy . y) over all rows; recomputes activations. */
int fdk_nn_backward(const float *params, const float *x, const float *dy, float *dparams, int64_t rows,
                    int32_t len, float scale, void *stream);
/* One Adam step (bias-corrected, step t >= 1) on n parameters. */
int fdk_adam_step(float *params, const float *grads, float *m, float *v, int64_t n, float lr, float beta1,
                  float beta2, float eps, int64_t t, void *stream);
/* Low-dose transmission data in place: p -> -log(max(Poisson(I0 exp(-mu p)), 1) / I0) / mu. */
int fdk_transmission_noise(float *dev_views, int64_t n, double i0, double mu, uint64_t seed, void *stream);
/* Ellipsoid phantom (records as fdk_phantom_project) sampled at voxel centres, [z][y][x]. */
int fdk_voxelize(const fdk_geometry *g, const double *ell, int32_t n_ell, float *dev_vol, void *stream);
/* ROWS views (n x nv x nu) -> MIRROR f32 pairs (n x nu x nv x 2), the staged backprojection's input. */
int fdk_rows_to_mirror(const float *dev_rows, void *dev_mirror, int64_t n_views, int32_t nu, int32_t nv,
                       void *stream);
/* Sum of squared errors of a backprojection volume ([x][y][z], as fdk_bp_volume_device of a full slab
 * pair) against truth ([z][y][x]) into *sse_host; dev_res (may be NULL) = 2 (vol - truth) / N, [z][y][x]. */
int fdk_volume_mse(const float *dev_vol_xyz, const float *dev_truth, float *dev_res, int32_t nx, int32_t ny,
                   int32_t nz, double *sse_host, void *stream);
/* Exact adjoint of the staged backprojection (FDK_BP_FP32 semantics) over the whole slab pair:
 * dev_grad (ROWS, n_views x nv x nu, accumulated) += BP^T(dev_res [z][y][x]).  dev_mats: device, 12
 * per view. */
int fdk_bp_adjoint(const fdk_geometry *g, const float *dev_res, const float *dev_mats, int32_t n_views,
                   float *dev_grad, void *stream);

/* ---- measurement probes (no reference counterpart) ------------------------ */
/* The backprojection is bound by shared-memory bandwidth or FP32 issue rate; these measure the
 * two denominators of its roofline on the given device: conflict-free 128-bit shared-memory
 * loads on every SM (GB/s) and independent FP32 FMA chains on every SM (TFLOP/s). */
int fdk_probe_smem(int32_t device, double *gbs);
int fdk_probe_fma(int32_t device, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* FDK_B200_FDK_H */
