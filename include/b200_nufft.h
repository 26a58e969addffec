/*
 * b200_nufft.h - device-pointer NUFFT plans on one NVIDIA B200 (sm_100a).
 *
 * This is the C ABI of libb200nufft.so that replaces the GPU-resident plan
 * API of wgpuNUFFT (src/plan.rs, src/type3.rs). wgpu buffers become CUDA
 * device pointers, a wgpu CommandEncoder becomes a CUDA stream, and the
 * queue order that executions of one plan must keep becomes stream order.
 * The host-array interface of the reference's C binding (wgpu_nufft_* and
 * wgpu_nufftf_*) is declared separately in wgpu_nufft.h and is exported by
 * the same library.
 *
 * Layouts follow the reference exactly:
 *   - coordinates are point-major: points[j * dim + axis], in radians, within
 *     [-3 pi, 3 pi] and periodic modulo 2 pi (src/plan.rs:750-762);
 *   - complex values are interleaved (re, im) pairs;
 *   - Fourier modes are stored axis-0 fastest, in centered order (index k of
 *     an axis of N modes holds frequency k - floor(N/2)) or FFT order;
 *   - a batch of B transforms sharing one point set is transform-major:
 *     c[b * M + j] and f[b * N + k] (src/config.rs:112-121).
 *
 * Definitions, with no normalization:
 *   type 1: f(k) = sum_j c(j) exp(i isign k.x(j))
 *   type 2: c(j) = sum_k f(k) exp(i isign k.x(j))
 *   type 3: f(k) = sum_j c(j) exp(i isign s(k).x(j))
 *
 * Every function returns a b200nufft_status; b200nufft_last_error() then
 * describes a failure on the calling thread. All device work is stream
 * ordered on the stream passed in (a cudaStream_t, passed as void*; NULL is
 * the legacy default stream). A plan may be used by one thread at a time, and
 * its executions must stay in stream order because they share the plan's
 * scratch memory, as the reference's executions share their fine grids
 * (src/plan.rs:452-456).
 */
#ifndef B200_NUFFT_H
#define B200_NUFFT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The names follow the variants of the reference's NufftError
 * (src/error.rs:8-200); the CUDA-specific ones replace the wgpu ones. */
typedef enum b200nufft_status {
  B200NUFFT_SUCCESS = 0,
  B200NUFFT_INVALID_BATCH = 1,              /* InvalidBatch */
  B200NUFFT_INVALID_DIMENSIONS = 2,         /* InvalidDimensions */
  B200NUFFT_ZERO_MODE = 3,                  /* ZeroMode */
  B200NUFFT_INVALID_TOLERANCE = 4,          /* InvalidTolerance */
  B200NUFFT_INVALID_SIGMA = 5,              /* InvalidSigma */
  B200NUFFT_KERNEL_WIDTH_UNSUPPORTED = 6,   /* KernelWidthUnsupported */
  B200NUFFT_F32_TOLERANCE_UNREACHABLE = 7,  /* F32ToleranceUnreachable */
  B200NUFFT_INVALID_KERNEL_WIDTH = 8,       /* InvalidKernelWidth */
  B200NUFFT_PRECISION_UNSUPPORTED = 9,      /* PrecisionUnsupported */
  B200NUFFT_INVALID_TYPE3_INTERVAL = 10,    /* InvalidType3Interval */
  B200NUFFT_TYPE3_GRID_SIZE_UNSUPPORTED = 11, /* Type3GridSizeUnsupported / VolumeUnsupported */
  B200NUFFT_TYPE3_RESCALING_UNSUPPORTED = 12, /* Type3RescalingUnsupported */
  B200NUFFT_LENGTH_OVERFLOW = 13,           /* LengthOverflow */
  B200NUFFT_INPUT_LENGTH = 14,              /* InputLength / CoordinateLength */
  B200NUFFT_FINE_GRID_MUST_BE_EVEN = 15,    /* FineGridMustBeEven */
  B200NUFFT_FINE_GRID_TOO_LARGE = 16,       /* FineGridTooLarge */
  B200NUFFT_FFT_SHAPE_UNSUPPORTED = 17,     /* FftShapeUnsupported */
  B200NUFFT_GPU_DIMENSIONS_UNSUPPORTED = 18,/* GpuDimensionsUnsupported */
  B200NUFFT_GPU_EXECUTION_UNAVAILABLE = 19, /* GpuExecutionUnavailable: wrong kind, no points */
  B200NUFFT_GPU_DEVICE_MISMATCH = 20,       /* GpuDeviceMismatch: another CUDA device is current */
  B200NUFFT_GPU_BUFFER_ALIAS_UNSUPPORTED = 21, /* GpuBufferAliasUnsupported */
  B200NUFFT_GPU_FINE_GRID_INDEX_UNSUPPORTED = 22, /* GpuFineGridIndexUnsupported */
  B200NUFFT_FFT_EXECUTION_FAILED = 23,      /* FftExecutionFailed (cuFFT) */
  B200NUFFT_INVALID_KERNEL_FOURIER_COEFFICIENT = 24, /* InvalidKernelFourierCoefficient */
  B200NUFFT_INVALID_ARGUMENT = 25,          /* a null pointer or an out-of-range option */
  B200NUFFT_DEVICE_ERROR = 26,              /* a CUDA runtime error */
  B200NUFFT_DEVICE_ALLOCATION_FAILED = 27,  /* cudaMalloc failed */
  B200NUFFT_DEVICE_TIMEOUT = 28,            /* a bounded device wait gave up */
  B200NUFFT_INTERNAL = 29
} b200nufft_status;

/* Precision of coordinates, values, window and FFT, numbered as the
 * reference's C interface numbers them (capi/include/wgpu_nufft.h:57-63).
 * F32: float coordinates and complex64 values. F64: double and complex128.
 * DF64: pairs of float words (hi, lo) per scalar, the reference's double-float
 * storage; B200 computes these plans in native f64. */
#define B200NUFFT_PRECISION_F64 1
#define B200NUFFT_PRECISION_DF64 2
#define B200NUFFT_PRECISION_F32 3

#define B200NUFFT_MODE_ORDER_CENTERED 0
#define B200NUFFT_MODE_ORDER_FFT 1

/* Type-1 and type-2 plans take 1 to 8 dimensions (4 to 8 run a generic
 * path without bins); type-3 plans 1 to 3. */
#define B200NUFFT_MAX_DIMENSIONS 8
#define B200NUFFT_MAX_TYPE3_DIMENSIONS 3

/* Type-1 spreading engines. AUTO runs 2D f32 type-1 plans of batch >= 16 on
 * the tensor cores (3xTF32 tcgen05 MMAs) when their active batch is at least
 * 16 and the chosen bins allow it, and everything else on the CUDA cores.
 * TENSOR_CORES asks for the tensor cores whenever the plan qualifies
 * (plan creation fails otherwise); CUDA_CORES never uses them. */
#define B200NUFFT_SPREAD_AUTO 0
#define B200NUFFT_SPREAD_CUDA_CORES 1
#define B200NUFFT_SPREAD_TENSOR_CORES 2

/* Mirror of NufftConfig (src/config.rs:66-229) plus the plan's type, the
 * CUDA device and the spreading engine. */
typedef struct b200nufft_config {
  int32_t type;        /* 1 or 2 */
  int32_t dimensions;  /* 1..B200NUFFT_MAX_DIMENSIONS */
  int64_t n_modes[8];  /* modes per axis, axis 0 first */
  int64_t batch;       /* most transforms per execution (with_batch), >= 1 */
  double eps;          /* tolerance, 0 < eps < 1 */
  int32_t isign;       /* >= 0 positive, < 0 negative (NufftSign::from_isign) */
  int32_t mode_order;  /* B200NUFFT_MODE_ORDER_* */
  double sigma;        /* upsampling factor, > 1; 0 selects 2 */
  int32_t precision;   /* B200NUFFT_PRECISION_*; 0 selects F32 */
  int32_t device;      /* CUDA device ordinal; -1 selects the current device */
  int32_t spread_method; /* B200NUFFT_SPREAD_*; no counterpart in the reference */
} b200nufft_config;

/* Fills *config with NufftConfig::default(): one mode, eps 1e-6, batch 1,
 * positive sign, centered order, sigma 2, F32, current device. */
void b200nufft_default_config(b200nufft_config *config);

typedef struct b200nufft_plan_s *b200nufft_plan;

/* Creates a type-1 or type-2 plan: NufftPlan::type1_gpu / type2_gpu
 * (src/plan.rs:457, src/plan.rs:606). Host work only plus device uploads of
 * the deconvolution amplitudes; scratch memory is reserved here and grows
 * on demand with larger point sets. */
int b200nufft_plan_create(const b200nufft_config *config, b200nufft_plan *plan);

/* Creates a plan without device resources: its metadata, buffer sizes and
 * kernel coefficients are available, executions fail with
 * B200NUFFT_GPU_EXECUTION_UNAVAILABLE. The analogue of the reference's
 * NufftPlan::type1 / type2 (src/plan.rs:449-455); needs no GPU. */
int b200nufft_plan_create_host(const b200nufft_config *config, b200nufft_plan *plan);

/* The bin geometry a point set of `point_count` points is binned with
 * (NdSpreadLayout::choose_geometry, src/gpu_nd_spread.rs:424-459), an index
 * into b200nufft_plan_info.geometry_sides. Type-1 plans; host only. */
int b200nufft_plan_choose_geometry(b200nufft_plan plan, int64_t point_count, int32_t *geometry);

/* Destroys a plan; a null plan is ignored. Synchronizes the plan's device. */
void b200nufft_plan_destroy(b200nufft_plan plan);

/* Plan metadata (NufftPlan::kernel, fine_grid_shape; src/plan.rs:700-715). */
typedef struct b200nufft_plan_info {
  int32_t type;
  int32_t dimensions;
  int32_t precision;
  int32_t kernel_width;
  double kernel_beta;
  int64_t fine_shape[8];
  int64_t mode_count;
  int64_t batch;
  /* Spreader bin geometries (NdSpreadLayout::for_grid, src/gpu_nd_spread.rs:194-407):
   * geometry_count sides of dimensions words each, finest first. */
  int32_t geometry_count;
  int32_t geometry_sides[16][8];
  /* Point set of the last b200nufft_set_points: its count and the geometry
   * it was binned with (NdSpreadLayout::choose_geometry), or -1. */
  int64_t point_count;
  int32_t chosen_geometry;
  int64_t bin_count;
} b200nufft_plan_info;

int b200nufft_plan_get_info(b200nufft_plan plan, b200nufft_plan_info *info);

/* Centered kernel Fourier coefficients phi_hat[k], k = 0..fine_shape[axis]/2,
 * with the (-1)^k grid-origin phase (NufftPlan::centered_kernel_fourier_coefficients,
 * src/plan.rs:717-724). `count` receives the number of values; `values` may be
 * null to query it. */
int b200nufft_plan_kernel_fourier_coefficients(b200nufft_plan plan, int32_t axis,
                                               double *values, int64_t capacity,
                                               int64_t *count);

/* Buffer sizes in bytes (src/plan.rs:732-794, 1032-1078). `active_batch`
 * must lie in 1..batch. */
int b200nufft_required_point_bytes(b200nufft_plan plan, int64_t point_count, uint64_t *bytes);
int b200nufft_required_input_bytes(b200nufft_plan plan, int64_t point_count,
                                   int64_t active_batch, uint64_t *bytes);
int b200nufft_required_output_bytes(b200nufft_plan plan, int64_t point_count,
                                    int64_t active_batch, uint64_t *bytes);

/* Prepares a point set for repeated executions (NufftPlan::set_points_gpu,
 * src/plan.rs:890-925): bins the points in a stable order and remembers the
 * device pointer, which must stay valid and unchanged until the next call.
 * point_count may be zero. */
int b200nufft_set_points(b200nufft_plan plan, int64_t point_count, const void *points,
                         void *stream);

/* Runs active_batch transforms on the remembered points
 * (NufftPlan::execute_type1_gpu_batch / execute_type2_gpu_batch,
 * src/plan.rs:946-977, 1197-1229). Type 1 reads `input` strengths (M per
 * transform) and overwrites every output mode; type 2 reads `input` modes and
 * writes `output` values (M per transform). `input` and `output` must not
 * overlap. With zero points a type-1 output is all zeros. */
int b200nufft_execute(b200nufft_plan plan, int64_t active_batch, const void *input,
                      void *output, void *stream);

/* b200nufft_set_points followed by b200nufft_execute: the reference's
 * encode_type1_gpu_batch / encode_type2_gpu_batch (src/plan.rs:836-872,
 * 1117-1139). */
int b200nufft_encode(b200nufft_plan plan, int64_t active_batch, int64_t point_count,
                     const void *points, const void *input, void *output, void *stream);

/* The stable bin order of the last set_points, for parity checks:
 * `permutation` (device, point_count words) receives the original index of
 * every slot and `bin_offsets` (device, bin_count + 1 words) the first slot of
 * every bin followed by the total (NdPointBins::encode,
 * src/gpu_nd_bins.rs:336-471). Either pointer may be null. 3D type-2 plans
 * interpolate in another order and sort the bin order at the first call after
 * each set_points, on `stream` (it reserves a device buffer of 3 coordinates
 * per point the first time). */
int b200nufft_copy_bin_order(b200nufft_plan plan, uint32_t *permutation,
                             uint32_t *bin_offsets, void *stream);

/* Waits until the plan's work on `stream` is done, then reports
 * B200NUFFT_DEVICE_TIMEOUT if a bounded device wait of the bin sort gave up
 * (its results are then invalid) and clears that flag. No counterpart in the
 * reference, whose plans never submit work themselves. */
int b200nufft_plan_synchronize(b200nufft_plan plan, void *stream);

/* Stage timing, the analogue of the reference's gpu-profiling stage layout
 * (src/gpu_profile.rs:12-120, NufftPlan::encode_type1_gpu_profiled,
 * src/plan.rs:990-1028). While enabled, set_points and execute record CUDA
 * events around every stage on the caller's stream; no host synchronization
 * is added. b200nufft_plan_stage_report() then, after the caller has
 * synchronized, sums the elapsed device time per stage over every recorded
 * launch and clears the record. */
#define B200NUFFT_STAGE_COUNT 12
/* Stage names, in report order. */
#define B200NUFFT_STAGE_NAMES \
  "bin_keys", "digit_scan", "radix_passes", "bin_offsets", "tile_parts", "strength_scale", \
  "spread", "fold", "fft", "deconvolution", "predeconvolution", "interpolation"

typedef struct b200nufft_stage_report {
  double milliseconds[B200NUFFT_STAGE_COUNT];
  int64_t launches[B200NUFFT_STAGE_COUNT];
} b200nufft_stage_report;

int b200nufft_plan_stage_timing(b200nufft_plan plan, int32_t enable);
int b200nufft_plan_stage_report(b200nufft_plan plan, b200nufft_stage_report *report);

/* The prepared slots of the reference's stable binning for the last
 * set_points (src/gpu_nd_bins.rs:590-709): per slot, `starts` (device,
 * (dim + 1) int32 words: the support start of every axis, then the original
 * index) and `offsets` (device, dim pairs of float words (hi, lo) holding
 * start - position). F32 plans only. */
int b200nufft_copy_prepared_slots(b200nufft_plan plan, int32_t *starts, float *offsets,
                                  void *stream);

/* Stable bin order without any device allocation. This entry point has no
 * counterpart in the reference. It is for callers that cannot call
 * cudaMalloc: code running while another framework owns every byte of device
 * memory through its own pool, and real-time or callback code where an
 * allocation may block or fail. It writes the same `permutation`
 * (point_count words) and `bin_offsets` (bins + 1 words, bins = prod_a
 * ceil(fine_shape[a] / bin_sides[a])) as b200nufft_set_points followed by
 * b200nufft_copy_bin_order on an F32 type-1 plan whose chosen bin geometry
 * has the sides `bin_sides` (b200nufft_plan_info.geometry_sides[chosen_geometry]);
 * `points` are point-major float coordinates. All scratch lives in a fixed
 * array of about 4.3 MB in the library's device image; point counts above
 * B200NUFFT_NOALLOC_MAX_POINTS are rejected with B200NUFFT_LENGTH_OVERFLOW.
 * The call allocates nothing: no cudaMalloc, no cudaFree, no library that
 * allocates. The CUDA driver places the array on a GPU when it loads the
 * library's module there: under lazy module loading (CUDA 12's default) at
 * this entry point's first call on that GPU, which looks up the array's
 * device address (cudaGetSymbolAddress, with that device current); with
 * CUDA_MODULE_LOADING=EAGER at the library's first use of the GPU. So make
 * that first call (a call with point_count 0 does this set-up and
 * only writes zero bin offsets) before
 * another framework takes the GPU's memory, and before any stream capture.
 * From then on the GPU holds the array until the process exits. Every call
 * shares the one array and starts by clearing what must start at zero, so
 * calls that overlap on the GPU (on different streams, or from different
 * threads) race and must be ordered by the caller. A sort whose look-back
 * wait gave up (bounded at about a second) writes 0xFFFFFFFF to
 * bin_offsets[bins], which otherwise equals point_count: check it after
 * synchronizing the stream. */
#define B200NUFFT_NOALLOC_MAX_POINTS 262144
int b200nufft_bin_order_noalloc(int32_t dimensions, const int64_t *fine_shape,
                                int32_t kernel_width, const int32_t *bin_sides,
                                int64_t point_count, const float *points, uint32_t *permutation,
                                uint32_t *bin_offsets, void *stream);

/* ------------------------------------------------------------------------ */
/* Type 3 (NufftType3Plan, src/type3.rs)                                     */
/* ------------------------------------------------------------------------ */

/* Mirror of NufftType3Config (src/type3.rs:100-213): conservative source
 * and target intervals per axis, every later coordinate must lie inside. */
typedef struct b200nufft_type3_config {
  int32_t dimensions;      /* 1..3 */
  int64_t batch;           /* most transforms per execution */
  double eps;
  int32_t isign;
  double sigma;            /* 0 selects 2 */
  int32_t precision;       /* B200NUFFT_PRECISION_*; 0 selects F64 */
  int32_t device;
  double source_lower[8];
  double source_upper[8];
  double target_lower[8];
  double target_upper[8];
} b200nufft_type3_config;

typedef struct b200nufft_type3_plan_s *b200nufft_type3_plan;

int b200nufft_type3_plan_create(const b200nufft_type3_config *config,
                                b200nufft_type3_plan *plan);
void b200nufft_type3_plan_destroy(b200nufft_type3_plan plan);

/* Type-3 metadata: the outer grid per axis and the inner type-2 fine grid. */
typedef struct b200nufft_type3_info {
  int32_t dimensions;
  int32_t kernel_width;
  double kernel_beta;
  int64_t outer_shape[8];
  int64_t inner_fine_shape[8];
  double source_center[8];
  double target_center[8];
  double gamma[8];
  double h[8];
} b200nufft_type3_info;

int b200nufft_type3_get_info(b200nufft_type3_plan plan, b200nufft_type3_info *info);

/* Sets M sources and N targets, both point-major device arrays in the plan's
 * precision, remembered until the next call. */
int b200nufft_type3_set_points(b200nufft_type3_plan plan, int64_t source_count,
                               const void *sources, int64_t target_count,
                               const void *targets, void *stream);

/* Runs active_batch transforms: `strengths` holds M values per transform and
 * `output` receives N values per transform. */
int b200nufft_type3_execute(b200nufft_type3_plan plan, int64_t active_batch,
                            const void *strengths, void *output, void *stream);

/* ------------------------------------------------------------------------ */

/* The message of the last failure on this thread; valid until the next call
 * on this thread. */
const char *b200nufft_last_error(void);

/* The library version. */
const char *b200nufft_version(void);

/* Many independent type-1 problems executed together. This has no
 * counterpart in the reference, which executes every plan on its own
 * (src/plan.rs). A batch holds 2D and 3D f32 type-1 plans of one window
 * width (one eps) on one device, each with its own grid and point set
 * (b200nufft_set_points before the first execution, which must not be
 * captured in a CUDA graph; later executions can be). An execution spreads
 * every problem's strengths from one persistent launch whose CTAs take
 * (problem, tile part) items from a device work counter, then runs each
 * problem's fold, FFT and deconvolution on streams forked from `stream` and
 * joined back to it. Every problem's modes are the bits of its own
 * execution. `strengths[p]` and `outputs[p]`: device buffers of problem p
 * (one vector). Executions of one batch stay in stream order. */
typedef struct b200nufft_batch_s *b200nufft_batch;
int b200nufft_batch_create(const b200nufft_plan *plans, int32_t count, b200nufft_batch *batch);
void b200nufft_batch_destroy(b200nufft_batch batch);
int b200nufft_batch_execute(b200nufft_batch batch, const void *const *strengths, void *const *outputs,
                            void *stream);

/* Launch choices of the type-1 spreader and the tensor-core paths. This has
 * no counterpart in the reference, which fixes them per rank and precision
 * (src/gpu_nd_spread.rs:55-135,562-593); here a table measured on a B200
 * (wgpunufft_b200/tune.py) holds them per workload key: plan type,
 * dimension, precision, window width, log2 of the fine-grid cells and log2
 * of the points per cell. Plans look the key up at set_points, so a key
 * always gets the same choices and outputs stay bitwise repeatable. */
typedef struct b200nufft_tuning {
  int32_t tile;                /* spreading tile side in cells (power of two) */
  int32_t ctas_per_sm;         /* CTAs per SM the tile parts are sized for */
  int32_t crowded_ctas_per_sm; /* the same on one-cell bins of >= 8 points per cell */
  int32_t tensor_min_batch;    /* smallest active batch on the tensor cores (AUTO) */
} b200nufft_tuning;

/* The choices the table gives a workload (type 1 or 2, B200NUFFT_PRECISION_*). */
int b200nufft_tuning_lookup(int32_t type, int32_t dimensions, int32_t precision, int32_t width,
                            int64_t fine_cells, int64_t point_count, b200nufft_tuning *out);

/* Process-wide override of the table for plans whose points are set later,
 * for the tuner's measurements; zero fields keep the table's choice, null
 * restores the table. Not for concurrent use with set_points. */
int b200nufft_tuning_override(const b200nufft_tuning *tuning);

/* Process-wide choice of the fine-grid transform of 2D and 3D f32 plans
 * created later: nonzero (the default) takes the fused shared-memory
 * transforms where every fine axis is a power of two from 64 to 4096 (one
 * pass per axis, pruned to the kept modes; type 1 folds in the first pass and
 * deconvolves in the last, type 2 predeconvolves in the first), zero takes
 * cuFFT for every plan. No counterpart in the reference, whose FFT is a
 * separate pass (wgpu-fft); for A/B comparisons. */
int b200nufft_set_fused_transforms(int enable);

/* Number of this library's kernel launches since the process started, for
 * accounting in benchmarks. */
uint64_t b200nufft_launch_count(void);

/* Tensor-core throughput on the current device (no counterpart in the
 * reference: the roofline of the tensor-core kernels). Every SM issues `iters`
 * back-to-back tcgen05 MMAs of M = 128, N = n (16 .. 256, a multiple of 16),
 * K = 8 (kind::tf32) or 16 (kind::f16 when f16 != 0) from one elected lane in
 * blocks of `unroll` (1, 4 or 16; iters a multiple of it), rotating over
 * `accumulators` accumulators (accumulators x n <= 256), A in tensor memory
 * when a_in_tmem, a commit every `commit_every` MMAs (0: at the end only).
 * Writes the launch's duration in milliseconds and, when cycles is not null,
 * SM cycles of CTA 0's issue loop and of issue plus drain. Returns 0, the
 * number of CTAs whose bounded wait gave up, or -1 on a CUDA error or bad
 * argument. Allocates a few bytes of device memory per call. */
int b200nufft_tf32_peak(int n, int a_in_tmem, int iters, int accumulators, int f16, int unroll, int commit_every,
                        float *ms, unsigned long long *cycles);

#ifdef __cplusplus
}
#endif

#endif /* B200_NUFFT_H */
