/*
 * wgpu_nufft.h - the host-array C interface of wgpuNUFFT, served by the B200
 * library (libb200nufft.so).
 *
 * These declarations restate the reference's C interface
 * (capi/include/wgpu_nufft.h:37-269) so that its Fortran, MATLAB and Julia
 * wrappers link against this library unchanged: same names, argument order,
 * array layouts and return codes. Plans take host arrays; points are copied to
 * the GPU at setpts and every execution copies its input to the GPU and its
 * output back, then returns.
 *
 * Array conventions, as in the reference: complex values interleaved (re, im);
 * Fourier modes axis 0 fastest, centered order unless the FFT order option is
 * set; batches of ntrans transforms one after another; type-1/2 coordinates in
 * [-3 pi, 3 pi]; no normalization; isign >= 0 is the positive sign.
 *
 * Differences from the reference: GPU plans run on a CUDA device (the one the
 * adapter options select, by CUDA ordinal order, name or PCI bus id); there is
 * no CPU engine, so WGPU_NUFFT_BACKEND_CPU is rejected with
 * WGPU_NUFFT_ERROR_PLAN and the automatic backend never falls back to the CPU.
 * Double-precision plans compute in native f64 on B200; WGPU_NUFFT_PRECISION_DF64
 * is honoured as the double-float storage format over the same f64 pipeline.
 */
#ifndef WGPU_NUFFT_H
#define WGPU_NUFFT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes (capi/include/wgpu_nufft.h:42-52). */
#define WGPU_NUFFT_SUCCESS 0
#define WGPU_NUFFT_ERROR_INVALID_ARGUMENT 1 /* null pointer, size, point out of range, call order */
#define WGPU_NUFFT_ERROR_PLAN 2             /* tolerance, dimensions, sizes or limits rejected */
#define WGPU_NUFFT_ERROR_GPU_UNAVAILABLE 3  /* no CUDA device, or no device that matches */
#define WGPU_NUFFT_ERROR_GPU 4              /* a CUDA or cuFFT error while running */
#define WGPU_NUFFT_ERROR_INTERNAL 5

/* Backends (capi/include/wgpu_nufft.h:54-57). */
#define WGPU_NUFFT_BACKEND_AUTO 0
#define WGPU_NUFFT_BACKEND_GPU 1
#define WGPU_NUFFT_BACKEND_CPU 2

/* Arithmetic (capi/include/wgpu_nufft.h:59-67). */
#define WGPU_NUFFT_PRECISION_AUTO 0
#define WGPU_NUFFT_PRECISION_F64 1
#define WGPU_NUFFT_PRECISION_DF64 2
#define WGPU_NUFFT_PRECISION_F32 3

#define WGPU_NUFFT_MODE_ORDER_CENTERED 0
#define WGPU_NUFFT_MODE_ORDER_FFT 1

#define WGPU_NUFFT_ADAPTER_NAME_SIZE 256
#define WGPU_NUFFT_PCI_BUS_ID_SIZE 32

/* Options; all zero selects every default (capi/include/wgpu_nufft.h:76-87). */
typedef struct wgpu_nufft_opts {
  int32_t backend;
  int32_t precision;
  int32_t mode_order;
  int32_t threads; /* accepted for compatibility; GPU plans ignore it */
  double sigma;    /* 0 selects 2 */
  int32_t adapter_index;
  char adapter_name[WGPU_NUFFT_ADAPTER_NAME_SIZE];
  char adapter_pci_bus_id[WGPU_NUFFT_PCI_BUS_ID_SIZE];
} wgpu_nufft_opts;

void wgpu_nufft_default_opts(wgpu_nufft_opts *opts);

/* One CUDA device per list entry (capi/include/wgpu_nufft.h:118-136). */
typedef struct wgpu_nufft_adapter {
  char name[WGPU_NUFFT_ADAPTER_NAME_SIZE];
  char backend[16];     /* "CUDA" */
  char device_type[16]; /* "DiscreteGpu" */
  char pci_bus_id[WGPU_NUFFT_PCI_BUS_ID_SIZE];
  int32_t is_default;
} wgpu_nufft_adapter;

int wgpu_nufft_list_adapters(wgpu_nufft_adapter *adapters, int32_t capacity, int32_t *count);

/* Extension with no counterpart in the reference: the adapter position
 * (0-based) that the selection fields of `opts` name in a given list of
 * adapter names and PCI bus ids (either may hold NULL entries; pci_bus_ids
 * may be NULL), with the reference's matching rules (capi/src/adapter.rs:
 * 175-207): names whole and case-insensitive, a PCI address without a
 * function matches every function, adapter_index counts the matches from 1,
 * and several matches without an index are an invalid argument. Returns 0,
 * WGPU_NUFFT_ERROR_INVALID_ARGUMENT or WGPU_NUFFT_ERROR_GPU_UNAVAILABLE. Lets
 * a host check a selection without a device; plans use the same rules over
 * the CUDA devices in ordinal order. */
int b200nufft_resolve_adapter(const char *const *names, const char *const *pci_bus_ids,
                              int32_t count, const wgpu_nufft_opts *opts, int32_t *position);
const char *wgpu_nufft_last_error(void);
const char *wgpu_nufft_version(void);
const char *wgpu_nufft_gpu_name(void);
void wgpu_nufft_shutdown(void);

/* Double precision (capi/include/wgpu_nufft.h:153-226). */
typedef struct wgpu_nufft_plan_s *wgpu_nufft_plan;

int wgpu_nufft_makeplan(int32_t type, int32_t dim, const int64_t *n_modes, int32_t isign,
                        int64_t ntrans, double eps, wgpu_nufft_plan *plan,
                        const wgpu_nufft_opts *opts);
int wgpu_nufft_setpts(wgpu_nufft_plan plan, int64_t M, const double *x, const double *y,
                      const double *z, int64_t N, const double *s, const double *t,
                      const double *u);
int wgpu_nufft_setpts_nd(wgpu_nufft_plan plan, int64_t M, const double *points, int64_t N,
                         const double *targets);
int wgpu_nufft_execute(wgpu_nufft_plan plan, double *c, double *f);
void wgpu_nufft_destroy(wgpu_nufft_plan plan);
int wgpu_nufft_plan_backend(wgpu_nufft_plan plan);
int wgpu_nufft_plan_precision(wgpu_nufft_plan plan);

int wgpu_nufft1d1(int64_t M, const double *x, const double *c, int32_t isign, double eps,
                  int64_t ms, double *f, const wgpu_nufft_opts *opts);
int wgpu_nufft1d2(int64_t M, const double *x, double *c, int32_t isign, double eps,
                  int64_t ms, const double *f, const wgpu_nufft_opts *opts);
int wgpu_nufft1d3(int64_t M, const double *x, const double *c, int32_t isign, double eps,
                  int64_t N, const double *s, double *f, const wgpu_nufft_opts *opts);
int wgpu_nufft2d1(int64_t M, const double *x, const double *y, const double *c, int32_t isign,
                  double eps, int64_t ms, int64_t mt, double *f, const wgpu_nufft_opts *opts);
int wgpu_nufft2d2(int64_t M, const double *x, const double *y, double *c, int32_t isign,
                  double eps, int64_t ms, int64_t mt, const double *f,
                  const wgpu_nufft_opts *opts);
int wgpu_nufft2d3(int64_t M, const double *x, const double *y, const double *c, int32_t isign,
                  double eps, int64_t N, const double *s, const double *t, double *f,
                  const wgpu_nufft_opts *opts);
int wgpu_nufft3d1(int64_t M, const double *x, const double *y, const double *z, const double *c,
                  int32_t isign, double eps, int64_t ms, int64_t mt, int64_t mu, double *f,
                  const wgpu_nufft_opts *opts);
int wgpu_nufft3d2(int64_t M, const double *x, const double *y, const double *z, double *c,
                  int32_t isign, double eps, int64_t ms, int64_t mt, int64_t mu,
                  const double *f, const wgpu_nufft_opts *opts);
int wgpu_nufft3d3(int64_t M, const double *x, const double *y, const double *z, const double *c,
                  int32_t isign, double eps, int64_t N, const double *s, const double *t,
                  const double *u, double *f, const wgpu_nufft_opts *opts);

/* Single precision (capi/include/wgpu_nufft.h:228-269). */
typedef struct wgpu_nufftf_plan_s *wgpu_nufftf_plan;

int wgpu_nufftf_makeplan(int32_t type, int32_t dim, const int64_t *n_modes, int32_t isign,
                         int64_t ntrans, double eps, wgpu_nufftf_plan *plan,
                         const wgpu_nufft_opts *opts);
int wgpu_nufftf_setpts(wgpu_nufftf_plan plan, int64_t M, const float *x, const float *y,
                       const float *z, int64_t N, const float *s, const float *t,
                       const float *u);
int wgpu_nufftf_setpts_nd(wgpu_nufftf_plan plan, int64_t M, const float *points, int64_t N,
                          const float *targets);
int wgpu_nufftf_execute(wgpu_nufftf_plan plan, float *c, float *f);
void wgpu_nufftf_destroy(wgpu_nufftf_plan plan);
int wgpu_nufftf_plan_backend(wgpu_nufftf_plan plan);
int wgpu_nufftf_plan_precision(wgpu_nufftf_plan plan);

int wgpu_nufftf1d1(int64_t M, const float *x, const float *c, int32_t isign, double eps,
                   int64_t ms, float *f, const wgpu_nufft_opts *opts);
int wgpu_nufftf1d2(int64_t M, const float *x, float *c, int32_t isign, double eps, int64_t ms,
                   const float *f, const wgpu_nufft_opts *opts);
int wgpu_nufftf1d3(int64_t M, const float *x, const float *c, int32_t isign, double eps,
                   int64_t N, const float *s, float *f, const wgpu_nufft_opts *opts);
int wgpu_nufftf2d1(int64_t M, const float *x, const float *y, const float *c, int32_t isign,
                   double eps, int64_t ms, int64_t mt, float *f, const wgpu_nufft_opts *opts);
int wgpu_nufftf2d2(int64_t M, const float *x, const float *y, float *c, int32_t isign,
                   double eps, int64_t ms, int64_t mt, const float *f,
                   const wgpu_nufft_opts *opts);
int wgpu_nufftf2d3(int64_t M, const float *x, const float *y, const float *c, int32_t isign,
                   double eps, int64_t N, const float *s, const float *t, float *f,
                   const wgpu_nufft_opts *opts);
int wgpu_nufftf3d1(int64_t M, const float *x, const float *y, const float *z, const float *c,
                   int32_t isign, double eps, int64_t ms, int64_t mt, int64_t mu, float *f,
                   const wgpu_nufft_opts *opts);
int wgpu_nufftf3d2(int64_t M, const float *x, const float *y, const float *z, float *c,
                   int32_t isign, double eps, int64_t ms, int64_t mt, int64_t mu,
                   const float *f, const wgpu_nufft_opts *opts);
int wgpu_nufftf3d3(int64_t M, const float *x, const float *y, const float *z, const float *c,
                   int32_t isign, double eps, int64_t N, const float *s, const float *t,
                   const float *u, float *f, const wgpu_nufft_opts *opts);

#ifdef __cplusplus
}
#endif

#endif /* WGPU_NUFFT_H */
