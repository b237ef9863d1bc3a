/*
 * s2dw_cuda.h -- C ABI of the B200 (sm_100a) implementation of the S2DW
 * directional scale-discretised wavelet transform on the sphere.
 *
 * Every entry point is a plain C function over plain pointers and sizes, so
 * that Fortran (ISO_C_BINDING), C, C++ and Python (ctypes) callers can bind
 * it directly.  Array arguments use the reference's Fortran column-major
 * layouts, first index fastest:
 *
 *   flm(0:B-1,0:B-1)                 complex128, flm[l + B*m]   (m <= l used)
 *   K_gamma(0:J,0:B-1)               float64,    K[j + (J+1)*l]
 *   Phi2(0:B-1)                      float64
 *   Slm(0:B-1,0:N-1)                 complex128, S[l + B*n]
 *   scoeff(0:bl_scoeff-1,0:bl_scoeff-1) complex128
 *   wav(0:J,0:2B-2,0:2B-1,0:N-1)     float64, static layout, scale fastest
 *   coeff_j(0:2bl-2,0:2bl-1,0:N-1)   float64, one array per scale j
 *                                    (the "dynamic" layout)
 *
 * Return values are status codes that mirror S2DW_ERROR_* of the reference
 * (src/mod/s2dw_error_mod.f90:37-52).  The reference prints and halts on a
 * fatal error; this library returns the code instead and keeps a message
 * for s2dwc_last_error_message().
 *
 * Host-buffer entry points are synchronous and allocate their device
 * workspace through a per-(B,N,alpha,J,device) plan cache.  The cached plan
 * keeps the tables folded from the caller's K_gamma, Slm and bl_scoeff while
 * later calls pass the same values (compared by content, so arrays changed
 * in place are picked up).  Their host<->device copies overlap the kernels a
 * scale at a time; page-locked per-scale arrays (cudaHostAlloc) copy at the
 * full PCIe rate, other arrays go through page-locked staging buffers of the
 * plan.  Device entry points (s2dwc_plan_*) take device pointers and a CUDA
 * stream and never synchronise.
 */
#ifndef S2DW_CUDA_H
#define S2DW_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: s2dw_error_mod.f90:37-52 */
#define S2DWC_OK 0
#define S2DWC_ERROR_INIT 1
#define S2DWC_ERROR_NOT_INIT 2
#define S2DWC_ERROR_INIT_FAIL 3
#define S2DWC_ERROR_MEM_ALLOC_FAIL 4
#define S2DWC_ERROR_ARTH 5
#define S2DWC_ERROR_ARTH_WARNING 6
#define S2DWC_ERROR_SIZE_WARNING 7
#define S2DWC_ERROR_SIZE_INVALID 8
#define S2DWC_ERROR_SIZE_NOT_DEF 9
#define S2DWC_ERROR_ARG_INVALID 10
#define S2DWC_ERROR_ARG_WARNING 11
#define S2DWC_ERROR_QUAD_STEP_EXCEED 12
#define S2DWC_ERROR_ADMISS_FAIL 13
#define S2DWC_ERROR_FILEIO 14
/* Not in the reference: a CUDA runtime call failed (device lost, launch
 * failure).  The message names the call. */
#define S2DWC_ERROR_CUDA 15

/* Precision form of the transform.  FP64: every stage in FP64, the drop-in
 * form.  SPLIT: the analysis and synthesis contractions run on the tensor
 * cores as exact int8 products of 48-bit fixed-point digits (six byte digits
 * per operand, per-row and per-column power-of-two scales, the 26 most
 * significant digit products summed exactly in int32), combined in FP64; the
 * d^l(pi/2) recurrences, the kernel tables and the beta/alpha transforms stay
 * FP64.  Its error is bounded by 1e-10 of max|w| per scale (analysis) and of
 * max|flm| (synthesis); it pays off for batches of maps
 * (s2dwc_plan_analysis_batch / _synthesis_batch), which share the d-operand. */
#define S2DWC_FORM_FP64 0
#define S2DWC_FORM_SPLIT 1

/* ---------------------------------------------------------------------- */
/* Library state                                                          */
/* ---------------------------------------------------------------------- */

/* Version string of this library. */
const char *s2dwc_version(void);

/* Optional explicit initialisation (CUDA context on the current device).
 * Host-buffer calls initialise lazily.  Returns S2DWC_OK. */
int s2dwc_init(void);

/* Frees every cached plan and its device memory. */
int s2dwc_finalize(void);

/* Text of a status code (the reference's error_comment table,
 * s2dw_error_mod.f90:58-76). */
const char *s2dwc_error_string(int code);

/* Detail of the last error raised on the calling thread. */
const char *s2dwc_last_error_message(void);

/* ---------------------------------------------------------------------- */
/* Kernel tables and helpers (host, FP64)                                 */
/* ---------------------------------------------------------------------- */

/* Replaces s2dw_core_assimilate_int, s2dw_core_mod.f90:1398-1415.
 * Returns 1 (assimilated, *y set) or 0 (*y = 0). */
int s2dwc_assimilate_int(double x, int *y);

/* Replaces s2dw_core_comp_Jmax, s2dw_core_mod.f90:1365-1376. */
int s2dwc_comp_jmax(int B, double alpha);

/* Per-scale band limits bl_hi, bl_lo of scale jj, the block repeated at
 * s2dw_core_mod.f90:372-381 / :607-616 / :850-859 / :1093-1102. */
int s2dwc_band_limits(int jj, int B, double alpha, int *bl_hi, int *bl_lo);

/* Number of doubles of scale jj's coefficient array (2bl-1)*2bl*N, the
 * shape allocated at s2dw_core_mod.f90:746. */
long long s2dwc_wav_scale_size(int jj, int B, int N, double alpha);

/* Replaces s2dw_core_init_kernels, s2dw_core_mod.f90:97-157. */
int s2dwc_init_kernels(double *K_gamma, double *Phi2, int *bl_scoeff, int J, int B, double alpha);

/* Replaces s2dw_core_init_directionality, s2dw_core_mod.f90:219-250. */
int s2dwc_init_directionality(double *Slm /* complex128 (B,N) */, int B, int N);

/* Replaces s2dw_core_admiss, s2dw_core_mod.f90:285-304.  *pass receives
 * 1 when every |admiss(l)-1| <= 1e-12. */
int s2dwc_admiss(double *admiss, const double *K_gamma, const double *Phi2, int B, int J, int *pass);

/* ---------------------------------------------------------------------- */
/* Transforms on host buffers (drop-in for the Fortran entry points)      */
/* ---------------------------------------------------------------------- */

/* Replaces s2dw_core_analysis_flm2wav, s2dw_core_mod.f90:342-534.
 * wav: static layout (J+1, 2B-1, 2B, N); only the region a<2bl-1, b<2bl
 * of each scale is written, as in the reference. */
int s2dwc_analysis_flm2wav(double *wav, double *scoeff, const double *flm, const double *K_gamma,
                           const double *Slm, int J, int B, int N, int bl_scoeff, double alpha);

/* Replaces s2dw_core_analysis_flm2wav_dynamic, s2dw_core_mod.f90:572-775.
 * wav_scales[jj] points at caller-owned storage of
 * s2dwc_wav_scale_size(jj,...) doubles (the Fortran shim allocates
 * wavdyn(jj)%coeff and passes c_loc of it). */
int s2dwc_analysis_flm2wav_dynamic(double *const *wav_scales, double *scoeff, const double *flm,
                                   const double *K_gamma, const double *Slm, int J, int B, int N,
                                   int bl_scoeff, double alpha);

/* Replaces s2dw_core_synthesis_wav2flm, s2dw_core_mod.f90:816-1019. */
int s2dwc_synthesis_wav2flm(double *flm, const double *wav, const double *scoeff,
                            const double *K_gamma, const double *Phi2, const double *Slm, int J,
                            int B, int N, int bl_scoeff, double alpha);

/* Replaces s2dw_core_synthesis_wav2flm_dynamic, s2dw_core_mod.f90:1060-1266.
 * The reference frees wavdyn; here the caller keeps ownership (the Fortran
 * shim deallocates after the call). */
int s2dwc_synthesis_wav2flm_dynamic(double *flm, const double *const *wav_scales,
                                    const double *scoeff, const double *K_gamma, const double *Phi2,
                                    const double *Slm, int J, int B, int N, int bl_scoeff,
                                    double alpha);

/* ---------------------------------------------------------------------- */
/* Device-resident API                                                    */
/* ---------------------------------------------------------------------- */

typedef struct s2dwc_plan s2dwc_plan;

/* Creates a plan for (B, N, alpha, J) on CUDA device `device`: cached
 * recurrence tables, chirp filters and workspaces.  `form` is
 * S2DWC_FORM_FP64 or S2DWC_FORM_SPLIT. */
int s2dwc_plan_create(s2dwc_plan **plan, int B, int N, double alpha, int J, int form, int device);
int s2dwc_plan_destroy(s2dwc_plan *plan);

/* Device bytes s2dwc_plan_create would allocate for (B, N, alpha, J, form),
 * computed on the host without touching a device (the split form's batch
 * workspaces, sized per batch later, are not included). */
int s2dwc_plan_footprint(int B, int N, double alpha, int J, int form, long long *bytes);

/* Limits the device memory one plan may hold to `bytes` (0: no limit, the
 * default; process-wide).  A plan whose footprint exceeds it is refused by
 * s2dwc_plan_create before any device call, and any later workspace growth
 * beyond it (split-form batches, host-buffer entry points) fails, both with
 * S2DWC_ERROR_MEM_ALLOC_FAIL -- the status the reference gives when an
 * allocate fails (src/mod/s2dw_core_mod.f90:384-385, :598-602).  The
 * host-buffer entry points create their plans through s2dwc_plan_create and
 * obey the same limit. */
int s2dwc_set_plan_memory_limit(long long bytes);

/* Uploads the caller's kernel tables (host pointers, reference layouts).
 * Phi2 may be NULL for analysis-only use.  Any complex Slm is accepted; one
 * not of the form s2dw_core_init_directionality produces (S/eta real, eta = 1
 * for odd N, i for even N) makes every FP64 contraction run twice, and the
 * split form refuses it (S2DWC_ERROR_ARG_INVALID). */
int s2dwc_plan_set_tables(s2dwc_plan *plan, const double *K_gamma, const double *Phi2,
                          const double *Slm, int bl_scoeff);

/* Packed per-scale wavelet layout used by the device API: scale jj starts
 * at offsets[jj] doubles and holds coeff_j in the dynamic layout;
 * offsets[J+1] is the total.  `offsets` has J+2 entries. */
int s2dwc_plan_wav_offsets(const s2dwc_plan *plan, long long *offsets);

/* Bytes of device workspace the plan holds. */
long long s2dwc_plan_workspace_bytes(const s2dwc_plan *plan);

/* Analysis on device memory.  d_wav: packed per-scale layout; d_scoeff:
 * (bl_scoeff, bl_scoeff) complex; d_flm: (B, B) complex.  `stream` is a
 * cudaStream_t (NULL = legacy default stream). */
int s2dwc_plan_analysis(s2dwc_plan *plan, double *d_wav, double *d_scoeff, const double *d_flm,
                        void *stream);

/* Synthesis on device memory (d_flm is overwritten). */
int s2dwc_plan_synthesis(s2dwc_plan *plan, double *d_flm, const double *d_wav,
                         const double *d_scoeff, void *stream);

/* Batches of maps with the same (B, N, alpha, J): map k's flm, packed
 * wavelets and scoeff start at k*B*B complex values, k*offsets[J+1] doubles
 * and k*bl_scoeff^2 complex values.  With S2DWC_FORM_SPLIT the analysis runs
 * the tensor-core contraction on groups of up to 32 maps; otherwise (and for
 * synthesis) the maps run one after another.  Not in the reference, whose
 * s2dw_wstats loops s2dw_core_analysis_flm2wav_dynamic over maps
 * (src/prog/s2dw_wstats.f90:181-197). */
int s2dwc_plan_analysis_batch(s2dwc_plan *plan, int nmaps, double *d_wav, double *d_scoeff,
                              const double *d_flm, void *stream);
int s2dwc_plan_synthesis_batch(s2dwc_plan *plan, int nmaps, double *d_flm, const double *d_wav,
                               const double *d_scoeff, void *stream);

/* Sizes the split form's map workspaces for batches of up to nmaps maps
 * (at most 32 are held; larger batches run in groups of 32).  The split
 * entry points grow these workspaces on demand, which frees the smaller ones:
 * a CUDA graph captured before a growth must not be replayed after it, and a
 * growth inside a capture fails with S2DWC_ERROR_ARG_INVALID.  Call this
 * before capturing batches.  Needs the kernel tables (s2dwc_plan_set_tables);
 * no effect in the FP64 form.  Not in the reference. */
int s2dwc_plan_reserve(s2dwc_plan *plan, int nmaps, void *stream);

/* Moments of the wavelet coefficients per scale for `nmaps` device-resident
 * maps in the packed layout (map k at d_wav + k*offsets[J+1]): the
 * computation of s2dw_stat_moments (src/mod/s2dw_stat_mod.f90:81-275) without
 * copying the coefficients to the host, as the reference's s2dw_wstats needs
 * (src/prog/s2dw_wstats.f90:181-197).  d_mask is one map's packed mask (the
 * same for every map) or NULL.  d_moments receives nmaps*(J+1)*6 doubles,
 * [map][scale][mean, var, skew, kur, five, six]; scales with zero variance
 * get zero higher moments, scales with fewer than two samples get zeros.
 * Unlike the reference, d_wav is not masked in place. */
int s2dwc_plan_stat_moments(s2dwc_plan *plan, int nmaps, const double *d_wav, const double *d_mask,
                            double *d_moments, void *stream);

/* Replaces s2dw_stat_moments, src/mod/s2dw_stat_mod.f90:81-275: host per-scale
 * arrays (the dynamic layout), the reference's argument order.  mask_scales,
 * five and six may be NULL (the reference's optional arguments); with a mask
 * the coefficients are masked in place, as in the reference.  Returns
 * S2DWC_ERROR_ARTH_WARNING (outputs written) when a scale has zero variance
 * and S2DWC_ERROR_SIZE_INVALID when one has fewer than two unmasked samples,
 * the reference's two error cases. */
int s2dwc_stat_moments(double *const *wav_scales, int J, int B, int N, double alpha, double *mean,
                       double *var, double *skew, double *kur, const double *const *mask_scales,
                       double *five, double *six);

/* Synchronises with the device and reports S2DWC_ERROR_CUDA if a split-form
 * kernel gave up waiting on its tensor-core pipeline since the last check
 * (the flag is cleared when reported); S2DWC_OK otherwise.  The outputs of
 * the calls that gave up are unspecified.  Failure detection of the kind
 * the reference's s2dw_error reports (src/mod/s2dw_error_mod.f90:127-191),
 * as a status instead of a halt. */
int s2dwc_plan_check(s2dwc_plan *plan);

/* Split-form plans: batches of fewer than `nmaps` maps run the FP64 path
 * (default 1: every batch runs the split contractions).  The split form
 * generates the Wigner-d digits once per batch, so it pays only from a
 * batch size on (about 17 maps at B=1024, N=4); a server that meets
 * batches of every size sets it to that crossover.  The results of a map
 * then depend on its batch's size, within the split form's 1e-10 bound.
 * No counterpart in the reference. */
int s2dwc_plan_set_split_min_batch(s2dwc_plan *plan, int nmaps);

/* CUDA stream priority of the plan's per-scale streams (CUDA's convention:
 * lower values run first; clamped to cudaDeviceGetStreamPriorityRange).  The
 * plan's kernels, and those of CUDA graphs captured from its calls after
 * this one, then take SMs ahead of work of lower priority: a server gives
 * its small, latency-bound transforms precedence over the full-band scales
 * of large ones.  Waits for the plan's streams to drain; call it between
 * transforms, outside stream capture.  No counterpart in the reference. */
int s2dwc_plan_set_priority(s2dwc_plan *plan, int priority);

/* Bound, in nanoseconds, on every wait of the split-form kernels' pipeline
 * (default 2 s).  A kernel whose wait runs out stops its work, lets its own
 * copies and tensor-core operations in flight finish, frees its tensor
 * memory and returns; s2dwc_plan_check then reports it.  A limit too short
 * for the pipeline's hand-offs (0 gives up on the first wait that is not
 * already satisfied) exercises that path in tests. */
int s2dwc_plan_set_wait_limit(s2dwc_plan *plan, long long ns);

/* Analysis on device memory that allocates nothing.  This entry point has no
 * counterpart in the reference.  It computes what s2dwc_plan_analysis
 * computes, with the same arguments, but takes its workspace (the F table and
 * one scale's Tg and Tb) from a fixed static device array of
 * S2DWC_NOALLOC_SCRATCH_BYTES instead of the plan's workspaces, and runs the
 * scales one after another on `stream`.  It makes no cudaMalloc, cudaFree or
 * other allocating call.  It is meant for callers that must not allocate
 * device memory once they are running: a program whose device memory is
 * already taken by its own pool allocator, or a loop in which an allocation
 * would synchronise the device and stall other streams.
 *  - Limit: the plan must need at most S2DWC_NOALLOC_SCRATCH_BYTES of scratch
 *    (16 (B B_pad + 3 N B^2) bytes, B_pad = B rounded up to a multiple of
 *    32, plus alignment): any B <= 256 with N <= 10, or B <= 512 with N <= 2.
 *    Larger plans are rejected with S2DWC_ERROR_SIZE_INVALID.
 *  - Form: the FP64 form only.  A plan created with S2DWC_FORM_SPLIT is
 *    rejected with S2DWC_ERROR_ARG_INVALID.
 *  - Setup: the first call on a device looks up the array's address
 *    (cudaGetSymbolAddress), which makes the CUDA driver load the module that
 *    holds it; make that first call during setup, before any stream capture.
 *    The address is cached per device until s2dwc_finalize.  A
 *    cudaDeviceReset unloads the module: call s2dwc_finalize after one, so
 *    that the next call looks the address up again.
 *  - Nothing needs to start at zero: each call writes every scratch element
 *    before it reads it.
 *  - There is one scratch array per device: calls that overlap in time on one
 *    device (different streams or host threads without ordering between them)
 *    race on it.  Order them on one stream or with events. */
#define S2DWC_NOALLOC_SCRATCH_BYTES (32LL << 20)
int s2dwc_plan_analysis_noalloc(const s2dwc_plan *plan, double *d_wav, double *d_scoeff,
                                const double *d_flm, void *stream);

/* Number of CUDA kernels one analysis / one synthesis launches. */
int s2dwc_plan_launch_count(const s2dwc_plan *plan, int *analysis, int *synthesis);

/* Per-kernel timing.  When enabled, the scales run one after another on the
 * caller's stream (instead of concurrently on the plan's streams) and every
 * launch is bracketed by CUDA events on that stream; s2dwc_plan_timing()
 * resolves the events (synchronising on them) and returns, for one kernel
 * kind, the launches and total device milliseconds accumulated since the
 * last reset. */
#define S2DWC_KIND_LWALK 0     /* analysis contraction + gamma DFT */
#define S2DWC_KIND_MWALK 1     /* synthesis contraction + harmonic sum */
#define S2DWC_KIND_ANA_BETA 2  /* analysis beta transform */
#define S2DWC_KIND_ANA_ALPHA 3 /* analysis alpha c2r transform */
#define S2DWC_KIND_SYN_ALPHA 4 /* synthesis alpha r2c transform */
#define S2DWC_KIND_SYN_BETA 5  /* synthesis gamma + beta transform and fold */
#define S2DWC_KIND_OTHER 6     /* scaling coefficients, zeroing */
#define S2DWC_KIND_COUNT 7
int s2dwc_plan_set_timing(s2dwc_plan *plan, int enable);
int s2dwc_plan_timing(s2dwc_plan *plan, int kind, long long *launches, double *total_ms);
int s2dwc_plan_timing_reset(s2dwc_plan *plan);

/* ---- Wavelet coefficient files (src/mod/s2dw_fileio_mod.f90) ----------
 * Host-side writers and readers of the reference's FITS and Matlab wavelet
 * files, so that coefficients computed here are read by the reference's
 * programs and the other way round.  Arguments keep the reference's order;
 * scoeff is complex128 (bl_scoeff x bl_scoeff), wav the static layout,
 * wav_scales the dynamic one.  Writers fail with S2DWC_ERROR_FILEIO if the
 * file exists, as the reference's do.  The reference's readers allocate
 * their outputs; here the caller reads the sizes with the _read_header
 * function first, allocates, and passes the same J, B, N, bl_scoeff to the
 * data reader (S2DWC_ERROR_SIZE_INVALID if they differ from the file's).
 * Readers report S2DWC_ERROR_FILEIO for a missing file, a wrong number of
 * HDUs, inconsistent sizes or null coefficients, the reference's checks. */

/* FITS: s2dw_fileio_fits_wav_write_dynamic, fileio:956-1079 */
int s2dwc_fileio_fits_wav_write_dynamic(double *const *wav_scales, const double *scoeff, int J, int B, int N,
                                        int bl_scoeff, double alpha, const char *filename, const char *comment);
/* FITS: s2dw_fileio_fits_wav_write_static, fileio:796-926 */
int s2dwc_fileio_fits_wav_write_static(const double *wav, const double *scoeff, int J, int B, int N, int bl_scoeff,
                                       double alpha, const char *filename, const char *comment);
/* The keywords s2dw_fileio_fits_wav_read_* start with (fileio:1325-1340). */
int s2dwc_fileio_fits_wav_read_header(const char *filename, int *J, int *B, int *N, int *bl_scoeff,
                                      double *alpha);
/* FITS: s2dw_fileio_fits_wav_read_dynamic, fileio:1286-1435 */
int s2dwc_fileio_fits_wav_read_dynamic(double *const *wav_scales, double *scoeff, int J, int B, int N,
                                       int bl_scoeff, const char *filename);
/* FITS: s2dw_fileio_fits_wav_read_static, fileio:1109-1253 */
int s2dwc_fileio_fits_wav_read_static(double *wav, double *scoeff, int J, int B, int N, int bl_scoeff,
                                      const char *filename);
/* Matlab: s2dw_fileio_matlab_wav_write_dynamic, fileio:298-436 (writes
 * filename, <base>_scoeff.dat and <base>_wcoeff.dat, base = filename
 * without ".m") */
int s2dwc_fileio_matlab_wav_write_dynamic(double *const *wav_scales, const double *scoeff, int J, int B, int N,
                                          int bl_scoeff, double alpha, const char *filename, const char *comment);
/* Matlab: s2dw_fileio_matlab_wav_write_static, fileio:102-268 */
int s2dwc_fileio_matlab_wav_write_static(const double *wav, const double *scoeff, int J, int B, int N,
                                         int bl_scoeff, double alpha, const char *filename, const char *comment);
/* The parameters s2dw_fileio_matlab_wav_read_* start with (fileio:660-680). */
int s2dwc_fileio_matlab_wav_read_header(const char *filename, int *J, int *B, int *N, int *bl_scoeff,
                                        double *alpha);
/* Matlab: s2dw_fileio_matlab_wav_read_dynamic, fileio:637-763 */
int s2dwc_fileio_matlab_wav_read_dynamic(double *const *wav_scales, double *scoeff, int J, int B, int N,
                                         int bl_scoeff, const char *filename);
/* Matlab: s2dw_fileio_matlab_wav_read_static, fileio:473-601 */
int s2dwc_fileio_matlab_wav_read_static(double *wav, double *scoeff, int J, int B, int N, int bl_scoeff,
                                        const char *filename);

#ifdef __cplusplus
}
#endif

#endif /* S2DW_CUDA_H */
