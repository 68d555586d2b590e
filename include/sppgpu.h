/*
 * sppgpu.h — C ABI of the B200 filterbank dedispersion library (libsppgpu.so).
 *
 * Plain C: pointers, sizes and status codes only.  Every entry point returns
 * an int status (SPP_OK == 0, negative on error) and, on error, leaves a
 * message for spp_last_error_string() in thread-local storage.
 *
 * Conventions
 *   - Unless stated otherwise every data pointer is a DEVICE pointer owned by
 *     the caller (e.g. a torch tensor's data_ptr()).  The "_host" entry points
 *     take host buffers and do their own copies.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Device work is stream-ordered; nothing synchronises unless the
 *     function says so.
 *   - Hot calls allocate nothing: scratch space ("workspace") is sized by the
 *     matching *_workspace_bytes() call and passed in by the caller.  Plans
 *     (spp_dmt_plan_*) allocate their device tables once at creation.
 *   - Filterbank input is the raw sigproc stream: time-major, `nchans`
 *     samples per spectrum, `nbits` in {1, 2, 4, 8} (packed, uint8 container)
 *     or 32 (float32).  `bitorder` is SPP_BITORDER_BIG or _LITTLE for packed
 *     data (sample k of a byte holds channel k of that byte's group).
 *
 * Each entry point names the reference interface it replaces
 * (FRBs/sigpyproc3, paths relative to src/sigpyproc/).
 */
#ifndef SPPGPU_H
#define SPPGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define SPP_OK 0
#define SPP_ERR_ARG (-1)         /* bad argument (null pointer, bad enum)       */
#define SPP_ERR_SIZE (-2)        /* buffer too small / shape inconsistent       */
#define SPP_ERR_ALIGN (-3)       /* pointer alignment requirement not met       */
#define SPP_ERR_CUDA (-4)        /* a CUDA runtime call failed                  */
#define SPP_ERR_TIMEOUT (-5)     /* a device-side bounded wait expired          */
#define SPP_ERR_UNSUPPORTED (-6) /* valid request outside what is implemented   */
#define SPP_ERR_DELAY (-7)       /* delay table out of the representable range  */
#define SPP_ERR_DEVICE (-8)      /* device status word reported an error        */

#define SPP_BITORDER_BIG 0
#define SPP_BITORDER_LITTLE 1

/* output element kinds */
#define SPP_OUT_F32 0 /* float32 samples                                       */
#define SPP_OUT_I32 1 /* int32 sums (integer input only; exact)                */
#define SPP_OUT_U16 2 /* uint16 sums, saturating (subband intermediates)       */

/* delay application modes for the DM-time transform */
#define SPP_MODE_DEDISPERSE 0 /* out[t] = sum_c x[t + d_c][c]   (kernels.dedisperse) */
#define SPP_MODE_ROLL 1       /* out[t] = sum_c x[(t - d_c) mod n][c] (kernels.dmt_block) */

/* float accumulation for float32 input */
#define SPP_ACC_KAHAN32 0 /* fp32 partial per slab of <= 32 channels, compensated
                             (Kahan 1965) sum across slabs                      */
#define SPP_ACC_F64 1     /* fp64 accumulator, as the reference kernels          */

const char* spp_last_error_string(void);
int spp_version(void);

/* Device status word helpers: kernels record bounded-wait timeouts and
 * defensive range checks in a 16-byte device status block (4 x uint32) that
 * lives at the start of every workspace.  spp_status_read copies it to
 * `host_out[4]` (synchronising `stream`) and returns SPP_OK, or SPP_ERR_DEVICE
 * if word 0 is non-zero. */
int spp_status_read(const void* workspace, uint32_t* host_out, void* stream);
int spp_status_clear(void* workspace, void* stream);

/* Page-lock (and release) host memory that already holds a filterbank, so
 * blocks are copied to the GPU by DMA straight from it instead of through a
 * staging buffer (the reference reads each block into a host buffer,
 * io/fileio.py:234-296; there is no device side to copy to).  A refused
 * registration (memory already registered, too large) returns SPP_ERR_CUDA
 * and leaves no pending CUDA error behind. */
int spp_host_register(void* ptr, int64_t bytes);
int spp_host_unregister(void* ptr);

/* ---- R4: unpack -------------------------------------------------------------
 * Replaces kernels.unpack{1,2,4}_8_{big,little} (core/kernels.py:20-69) and
 * io/bits.py unpack (:19-70): `nbytes` packed bytes -> nbytes*8/nbits uint8
 * samples, sample k of byte i written to out[i*8/nbits + k]. */
int spp_unpack(const uint8_t* in, int64_t nbytes, int nbits, int bitorder,
               uint8_t* out, void* stream);

/* ---- R2: single-DM dedispersion ---------------------------------------------
 * Replaces kernels.dedisperse / dedisperse_par (core/kernels.py:340-362, :542):
 *   out[out_start + t] = sum_c x[t + delays[c]][c],  t < nsamps - max|delays|
 * with negative row indices wrapping within the block (numba semantics).
 * Integer input is summed exactly; float32 input with `acc` (SPP_ACC_F64
 * matches the reference's float64 accumulator).  `delays` is a device int32
 * array of nchans entries; delay_min/delay_max are its min and max (the host
 * knows them; the kernel range-checks every entry against them).
 * `out_len` is the full length of `out`; the call fails with SPP_ERR_SIZE if
 * out_start + nsamps - max|d| > out_len (the reference has no such check). */
int64_t spp_dedisperse_workspace_bytes(int nbits, int64_t nchans, int64_t nsamps,
                                       int32_t delay_min, int32_t delay_max);
int spp_dedisperse(const void* in, int nbits, int bitorder, int64_t nchans,
                   int64_t nsamps, const int32_t* delays, int32_t delay_min,
                   int32_t delay_max, float* out, int64_t out_len,
                   int64_t out_start, int acc, void* workspace,
                   int64_t workspace_bytes, void* stream);

/* The same computation for 8-bit data with `delays_host` in HOST memory -- the
 * form kernels.dedisperse(in, out, delays, nchans, nsamps, out_start) takes it
 * (core/kernels.py:340-347).  Knowing the delays on the host lets the call
 * precompute every row range and channel offset into the kernel's parameters
 * (one launch, no workspace, no delay upload; a CUDA graph that captures the
 * call records the parameters).  Returns SPP_ERR_UNSUPPORTED (nothing
 * launched) unless
 * nbits == 8, nchans is a multiple of 32 and at most 1024, `in` is 16-B
 * aligned and the block's slabs fit in shared memory together; callers then
 * use spp_dedisperse. */
int spp_dedisperse_hd(const void* in, int nbits, int64_t nchans, int64_t nsamps,
                      const int32_t* delays_host, float* out, int64_t out_len,
                      int64_t out_start, void* stream);

/* ---- folding -------------------------------------------------------------
 * Replaces kernels.fold (core/kernels.py:403-445) for one read_plan block
 * (Filterbank.fold, base.py:1109-1207): sample t of the block (t < nsamps -
 * maxdelay, global time index + t) of channel c, read at row t + delays[c],
 * is added into fold_ar[(subint * nsubs + band) * nbins + phasebin] and
 * counted in count_ar, with the reference's float64 phase arithmetic on the
 * float32 tsamp / period / accel it receives and Python's float floor
 * division for the subintegration.  `band_start` (device, nsubs + 1 int32)
 * gives each subband's first channel as the reference's `ichan // (nchans /
 * nsubs)` assigns them.  `in`: time-major uint8 (nbits 8) or float32 (nbits
 * 32) on the device; fold_ar / count_ar (device, `cells` >= nints * nsubs *
 * nbins entries) accumulate across calls.  uint8 sums are exact while a cell
 * stays below 2^24, hence equal to the reference's float32 cells; float32
 * sums differ from its sequential adds by rounding only. */
int spp_fold(const void* in, int nbits, int64_t nchans, int64_t nsamps,
             const int32_t* delays, int32_t maxdelay, float tsamp, float period,
             float accel, int64_t total_nsamps, int32_t nbins, int32_t nints,
             int32_t nsubs, int64_t index, const int32_t* band_start, float* fold_ar,
             int32_t* count_ar, int64_t cells, void* stream);
/* The 8-bit form with exact cells: fold_sums holds 64-bit integer sums (the
 * caller converts them to float32 once at the end), so the result is exact and
 * independent of the order of the atomic adds for any observation length.
 * The reference's float32 cells (sequential adds) equal it while every cell
 * stays below 2^24. */
int spp_fold_exact(const void* in, int64_t nchans, int64_t nsamps,
                   const int32_t* delays, int32_t maxdelay, float tsamp,
                   float period, float accel, int64_t total_nsamps,
                   int32_t nbins, int32_t nints, int32_t nsubs, int64_t index,
                   const int32_t* band_start, unsigned long long* fold_sums,
                   int32_t* count_ar, int64_t cells, void* stream);

/* Same computation as spp_dedisperse, but allocating nothing and taking no
 * workspace.  No counterpart in the reference.  It serves callers that must not
 * allocate device memory while running (a real-time pipeline that reserves its
 * memory at start-up and treats a later cudaMalloc -- which may synchronise the
 * device or fail under memory pressure -- as an error, or a host framework whose
 * allocator owns device memory and hands out only input and output buffers).
 * Its scratch is a fixed array of spp_dedisperse_noalloc_max_bytes() (32 MiB)
 * compiled into the library, which every GPU that loads the library holds until
 * the process exits; blocks whose scratch would exceed it are rejected with
 * SPP_ERR_SIZE.  The first call on each device looks the array up with
 * cudaGetSymbolAddress, so make that first call before any stream capture.
 * All calls share the one array and leave the last call's data in it: calls
 * that can overlap on the GPU (different streams, or several host threads)
 * race with each other and must be serialised by the caller. */
int64_t spp_dedisperse_noalloc_max_bytes(void);
int spp_dedisperse_noalloc(const void* in, int nbits, int bitorder, int64_t nchans,
                           int64_t nsamps, const int32_t* delays, int32_t delay_min,
                           int32_t delay_max, float* out, int64_t out_len,
                           int64_t out_start, int acc, void* stream);
/* The device status words of the last spp_dedisperse_noalloc call on the
 * current device (they live in the fixed array, which the caller cannot
 * address): copies the 4 words to host_out[4], synchronising `stream`, and
 * returns SPP_ERR_DEVICE if word 0 is non-zero -- a bounded wait ran out
 * (SPP_DEV_TIMEOUT, the output is incomplete) or a delay lay outside the
 * declared [delay_min, delay_max] and was clamped (SPP_DEV_RANGE, the output
 * is wrong).  Each spp_dedisperse_noalloc call clears the words first.  No
 * counterpart in the reference. */
int spp_dedisperse_noalloc_status_read(uint32_t* host_out, void* stream);

/* ---- R3: DM-trial batch (DM-time transform) -----------------------------------
 * Replaces FilterbankBlock.dmt_transform (block.py:309-343) / kernels.dmt_block
 * (core/kernels.py:1155-1168).  A plan owns the ndm x nchans delay table on the
 * device and the tile geometry; execute runs
 *   SPP_MODE_DEDISPERSE: out[i][t] = sum_c x[t + D[i][c]][c], t < nsamps - max|D|
 *   SPP_MODE_ROLL:       out[i][t] = sum_c x[(t - D[i][c]) mod nsamps][c], t < nsamps
 * writing rows of `out` with row stride `out_stride` elements starting at
 * column `out_start`.  delays_host is a host int32 array (ndm x nchans,
 * row-major), read once at plan creation. */
typedef struct spp_dmt_plan spp_dmt_plan;
int spp_dmt_plan_create(spp_dmt_plan** plan, int nbits, int bitorder,
                        int64_t nchans, int64_t nsamps_max, int64_t ndm,
                        const int32_t* delays_host, int mode, int out_kind,
                        int acc);
int spp_dmt_plan_destroy(spp_dmt_plan* plan);
/* valid output samples per row for an input of `nsamps` samples */
int64_t spp_dmt_plan_nvalid(const spp_dmt_plan* plan, int64_t nsamps);
int64_t spp_dmt_plan_workspace_bytes(const spp_dmt_plan* plan, int64_t nsamps);
/* describe the chosen tiles: fills cfg[8] = {nbits | 256 * bit_sliced |
 * 512 * paired, R, DW, TW, SLAB, STAGES, T (samples per tile), smem bytes};
 * bit_sliced = 1 when the kernel counts over bit-plane rows (R = words per
 * thread); paired = 1 for the 2-bit channel-pair kernels (SLAB counts pairs;
 * the workspace then also holds one three-plane row per pair and relative
 * delay, which spp_dmt_plan_workspace_bytes includes) */
int spp_dmt_plan_describe(const spp_dmt_plan* plan, int32_t* cfg);
/* override the tile shape (autotuner); variant index in [0, n) */
int spp_dmt_plan_num_variants(const spp_dmt_plan* plan);
int spp_dmt_plan_set_variant(spp_dmt_plan* plan, int variant);
/* Per-kernel device timing: while enabled, each execute records CUDA events on
 * its stream around the corner turn and the DM-time kernel;
 * spp_dmt_plan_timing_read synchronises them and returns the summed
 * milliseconds and the number of executions since enabling. */
int spp_dmt_plan_timing(spp_dmt_plan* plan, int enable);
int spp_dmt_plan_timing_read(spp_dmt_plan* plan, double* ms_corner_turn,
                             double* ms_dmt, int32_t* nexec);
int spp_dmt_execute(const spp_dmt_plan* plan, const void* in, int64_t nsamps,
                    void* out, int64_t out_stride, int64_t out_start,
                    void* workspace, int64_t workspace_bytes, void* stream);
/* Float32 input with the zero-DM filter of kernels.remove_zerodm
 * (core/kernels.py:465-505) fused into the load: every sample becomes
 * f32((f64(x) - zdm[t]*f64(chanwts[c])) + f64(bpass[c])), zdm[t] = sum_c f64(x[t][c]),
 * before the transform.  bpass/chanwts are device float arrays (nchans). */
int64_t spp_dmt_plan_zero_dm_workspace_bytes(const spp_dmt_plan* plan, int64_t nsamps);
int spp_dmt_execute_zero_dm(const spp_dmt_plan* plan, const float* in, int64_t nsamps,
                            const float* bpass, const float* chanwts, void* out,
                            int64_t out_stride, int64_t out_start, void* workspace,
                            int64_t workspace_bytes, void* stream);
/* Same transform end to end from HOST memory: `in_host` (pinned or pageable)
 * and `out_host` (ndm x out_stride elements).  Time is cut into blocks of
 * `block_nsamps` output samples; H2D, compute and D2H of successive blocks
 * overlap on three internal streams.  Synchronous: returns when out_host is
 * complete. */
int spp_dmt_execute_host(const spp_dmt_plan* plan, const void* in_host,
                         int64_t nsamps, void* out_host, int64_t out_stride,
                         int64_t block_nsamps, void* workspace,
                         int64_t workspace_bytes);
int64_t spp_dmt_host_workspace_bytes(const spp_dmt_plan* plan,
                                     int64_t block_nsamps);

/* ---- R10 / N2: channel statistics and zero-DM --------------------------------
 * spp_bandpass: kernels.extract_bpass (core/kernels.py:281-292): bpass[c] +=
 * sum_t x[t][c], accumulated sequentially in float32 per channel exactly as the
 * reference loop (bit-identical).  spp_collapse: kernels.extract_tim
 * (core/kernels.py:255-278): tim[out_start + t] += sum_c x[t][c] (float64
 * accumulator, stored float32).  spp_zero_dm: kernels.remove_zerodm
 * (core/kernels.py:465-505) for float32 input:
 *   y[t][c] = f32((f64(x) - zdm[t] * f64(bpass[c]/sum(bpass))) + f64(bpass[c]))
 * with zdm[t] = sum_c f64(x[t][c]); `chanwts` is bpass/sum(bpass) computed by
 * the caller in float32 (as the reference). */
int spp_bandpass(const void* in, int nbits, int bitorder, int64_t nchans,
                 int64_t nsamps, float* bpass, void* stream);
int spp_collapse(const void* in, int nbits, int bitorder, int64_t nchans,
                 int64_t nsamps, float* tim, int64_t out_start, void* stream);
int spp_zero_dm(const float* in, float* out, int64_t nchans, int64_t nsamps,
                const float* bpass, const float* chanwts, void* stream);
/* The same for uint8 input (8-bit files, Filterbank.remove_zerodm
 * base.py:961-1028): each value stored as the low eight bits of the truncated
 * float64 result, which is what the reference's numba cast to uint8 writes
 * (the bandpass term is a channel sum, far above 255). */
int spp_zero_dm_u8(const uint8_t* in, uint8_t* out, int64_t nchans,
                   int64_t nsamps, const float* bpass, const float* chanwts,
                   void* stream);

/* ---- R8: downsample ----------------------------------------------------------
 * kernels.downsample_1d_mean (core/kernels.py:176-204): out[i] =
 * f32(sum_{k<factor} f64(in[i*factor+k]) / factor) for i < n / factor, for
 * `nrows` independent rows of `n` samples (row strides in elements). */
int spp_downsample_mean(const float* in, int64_t nrows, int64_t n,
                        int64_t in_stride, int factor, float* out,
                        int64_t out_stride, void* stream);
/* kernels.downsample_2d_mean_flat (core/kernels.py:207-252): a dim1 x dim2
 * row-major block (dim2 fastest) -> (dim1/factor1) x (dim2/factor2) means of
 * factor1 x factor2 cells (float64 sums; the remainders dropped).  The _u8
 * form keeps uint8 output as the reference does for 8-bit data (the mean
 * truncated toward zero). */
int spp_downsample_2d_mean(const float* in, int64_t dim1, int64_t dim2,
                           int factor1, int factor2, float* out, void* stream);
int spp_downsample_2d_mean_u8(const uint8_t* in, int64_t dim1, int64_t dim2,
                              int factor1, int factor2, uint8_t* out,
                              void* stream);

/* ---- R9: boxcar matched filter -> S/N peaks ------------------------------------
 * For each of `nrows` rows (row stride `in_stride` elements, `n` valid samples,
 * element kind in_kind = SPP_OUT_F32 or SPP_OUT_I32), for each downsample
 * factor f in factors[0..nfactors) and boxcar width w in widths[0..nwidths)
 * (HOST arrays; nfactors <= 8, nwidths <= 32, 1 <= w <= 4096):
 *   y = downsample_1d_mean(row, f)   (length n_f = n / f)
 *   mean, std = of y (float64, population std)
 *   snr = max_{t <= n_f - w} (sum_{k<w} y[t+k] - w*mean) / (std * sqrt(w))
 * written to snr[row][fi][wi] (float32) and, if `peak_index` is not NULL, the
 * argmax t to peak_index[row][fi][wi] (int32).  Semantics follow
 * TimeSeries.downsample + apply_boxcar (timeseries.py:107-132, :296-325) on a
 * z-scored series (stats.estimate_zscore, core/stats.py:418-477, loc=mean,
 * scale=std). */
int64_t spp_boxcar_snr_workspace_bytes(int64_t nrows, int64_t n, int nfactors,
                                       int nwidths);
int spp_boxcar_snr(const void* in, int in_kind, int64_t nrows, int64_t n,
                   int64_t in_stride, const int32_t* factors, int nfactors,
                   const int32_t* widths, int nwidths, float* snr,
                   int32_t* peak_index, void* workspace,
                   int64_t workspace_bytes, void* stream);
/* TimeSeries.apply_boxcar (timeseries.py:296-325) with stats.running_filter
 * "mean" (core/stats.py:200-243): out[(i + ref_bin) mod n] = f32(sqrt(w) *
 * mean(p[i .. i+w-1])), p = the n samples padded symmetrically (np.pad
 * "symmetric") by w/2 on the left and w/2 (odd w) or w/2-1 (even w) on the
 * right, ref_bin = -floor(w/2) (the reference's -w // 2 + 1 for odd w, -w // 2
 * for even w, in Python floor division).  Window sums in float64
 * (the reference's bottleneck.move_mean keeps a float32 running sum).
 * 1 <= width <= 8192; `in` and `out` distinct device arrays of n floats. */
int spp_boxcar_filter(const float* in, int64_t n, int width, float* out,
                      void* stream);

/* The same with the robust location and scale of the reference MatchedFilter's
 * defaults (core/filters.py:105-125: stats.estimate_zscore with loc_method
 * "median", scale_method "iqr", core/stats.py:418-502): per row and factor,
 *   loc   = median of y (float32; the two middle values averaged in float32)
 *   scale = (q75 - q25) / 1.3489795003921634 (float64; numpy's linear
 *           percentile interpolation; 1 when ~0)
 *   snr   = max_t (sum_{k<w} y[t+k] - w*loc) / (scale * sqrt(w)).
 * The order statistics are exact (radix selection over the float32 y). */
int64_t spp_boxcar_snr_robust_workspace_bytes(int64_t nrows, int64_t n,
                                              int nfactors, int nwidths);
int spp_boxcar_snr_robust(const void* in, int in_kind, int64_t nrows,
                          int64_t n, int64_t in_stride, const int32_t* factors,
                          int nfactors, const int32_t* widths, int nwidths,
                          float* snr, int32_t* peak_index, void* workspace,
                          int64_t workspace_bytes, void* stream);

/* ---- N3: matched filter -------------------------------------------------------
 * MatchedFilter (core/filters.py:29-365) on the GPU.
 * spp_row_loc_scale: per row of `nrows` (row stride `in_stride` elements, n
 * samples, in_kind SPP_OUT_F32 / SPP_OUT_I32), the (loc, scale) pair of
 * stats.estimate_zscore (core/stats.py:418-502) into loc_scale[row * 2 + 0/1]
 * (device float64): method 0 = mean / population std, method 1 = median
 * (float32, the two middle values averaged in float32) / IQR / 1.349 (exact
 * order statistics), method 2 = the same median / stats._scale_mad
 * (core/stats.py:505-536: median absolute deviation from the float64 median
 * / 0.6745, exact order statistics; the mean absolute deviation / sqrt(2/pi)
 * when that is within 1e-8 of 0); a scale within 1e-8 of 0 becomes 1.
 * spp_zscore: out[i] = f32(f64(f32(in[i] - f32(loc))) / scale), the rounding
 * of np.subtract(..., dtype=float32) then np.divide into float32.
 * spp_matched_filter: kernels.convolve_templates (core/kernels.py:861-906)
 * for the z-scored series z of n samples and FFT length nfft >= n
 * (pocketfft's good size for real transforms, as the reference asks
 * rocket_fft for): for template k (float64 samples temps[temp_offsets[k] ..
 * temp_offsets[k+1]), reference bin ref_bins[k]) and t < n,
 *   convs[k * n + t] = (sum_j h[j] z[((t + j - ref) mod nfft) mod n]
 *                       - mu_k * sum_{m < nfft} z[m mod n]) / sigma_k
 * with temp_stats[2k .. 2k+1] = (mu_k, sigma_k) = (sum h / nfft,
 * sqrt(sum h^2 - (sum h)^2 / nfft)): the circular correlation with the
 * template zero-padded to nfft, reference bin at 0, normalised to zero mean
 * and unit power, that the reference computes by FFT; here direct, float64.
 * The workspace (>= 16 B, device) receives sum z (float64) and, in its
 * second 8 bytes, the first maximum of convs in (template, sample) order as
 * an unsigned 64-bit key: high word the float's order-preserving bits, low
 * word 0xFFFFFFFF - flat index. */
int spp_row_loc_scale(const void* in, int in_kind, int64_t nrows, int64_t n,
                      int64_t in_stride, int method, double* loc_scale,
                      void* stream);
int spp_zscore(const float* in, int64_t n, const double* loc_scale, float* out,
               void* stream);
int spp_matched_filter(const float* z, int64_t n, int64_t nfft,
                       const double* temps, const int32_t* temp_offsets,
                       const int32_t* ref_bins, const double* temp_stats,
                       int ntemps, float* convs, void* workspace,
                       int64_t workspace_bytes, void* stream);

/* ---- R7: subband dedispersion ----------------------------------------------------
 * Stage 1 replaces kernels.subband (core/kernels.py:379-401) with a zeroed
 * output: out[t][s] = sum_{c: chan_to_sub[c]==s} x[t + delays[c]][c] for
 * t < nsamps - maxdelay, (nsamps - maxdelay) x nsub float32, row-major.
 * `delays` and `chan_to_sub` are device int32 arrays of nchans entries. */
int spp_subband(const void* in, int nbits, int bitorder, int64_t nchans,
                int64_t nsamps, const int32_t* delays, int32_t maxdelay,
                const int32_t* chan_to_sub, int64_t nsub, float* out,
                void* stream);

/* ---- Batched / persistent DM-time transform (many beams, chunks, DM ranges) -------
 * One persistent launch processes a work list of items; each item is one DM
 * tile (nrows <= DW trial rows) x one time tile of T samples starting at t0, with
 * its own planar rows, delay rows and output rows, so beams of different
 * lengths, channel groups (subbands) and DM ranges share a launch.  Items are
 * claimed from `counter` (reset by the launch), tiles come from
 * spp_wl_describe.  Planar rows are produced by spp_corner_turn (layout from
 * spp_planar_layout) or are the uint16 rows of a previous SPP_OUT_U16 pass
 * (nbits = 16).  No reference counterpart: the reference runs one DM of one
 * file per call (kernels.dedisperse, core/kernels.py:340-362). */
typedef struct spp_dmt_item {
  const void* planar;     /* first planar row of the channel group           */
  int64_t pitch_w;        /* 32-bit words per planar row                     */
  int64_t halo;           /* left halo (samples) of the planar rows          */
  const int32_t* delays;  /* delay row of the tile's first DM                */
  int64_t dpitch;         /* elements between delay rows                     */
  void* out;              /* output row of the tile's first DM               */
  int64_t out_stride;     /* elements between output rows                    */
  int64_t out_start;      /* element offset of sample 0 within a row         */
  int64_t nvalid;         /* samples to write per row                        */
  int64_t t0;             /* first output sample of this tile                */
  int32_t nchans;         /* channels in the group                           */
  int32_t nrows;          /* DM rows in this tile (<= DW)                    */
  int32_t sign;           /* +1: x[t + d], -1: x[t - d]                      */
  int32_t dlo, dhi;       /* range of sign*delay (checked on the device)     */
  int32_t span_max;       /* max over channels of the tile's delay spread    */
  int32_t out_kind;       /* SPP_OUT_F32 / _I32 / _U16                       */
  int32_t reserved;
} spp_dmt_item;           /* 112 bytes */

int spp_wl_num_variants(int nbits, int acc);
/* cfg[8] = {R, DW, TW, SLAB, STAGES, T (samples per item), threads,
 *           samples per word | 256 if the variant is bit-sliced} */
int spp_wl_describe(int nbits, int acc, int variant, int32_t* cfg);
int32_t spp_wl_slot_words(int nbits, int acc, int variant, int32_t span_max);
int64_t spp_wl_smem_bytes(int nbits, int acc, int variant, int32_t slot_w);
/* nctas <= 0: one wave of resident CTAs.  `items` is a device array. */
int spp_wl_launch(int nbits, int acc, int variant, const void* items, int32_t nitems,
                  int32_t slot_w, int32_t* counter, uint32_t* status, int32_t nctas,
                  void* stream);
/* CTAs of one resident wave for a variant (sets its shared-memory limit). */
int32_t spp_wl_default_ctas(int nbits, int acc, int variant, int32_t slot_w);
/* Planar layout for offsets in [omin, omax] and nvalid outputs tiled by tile_T. */
int spp_planar_layout(int nbits, int64_t tile_T, int64_t nvalid, int32_t omin,
                      int32_t omax, int32_t slot_w, int64_t* halo, int64_t* pitch_w);
/* Planar layout and corner turn matching a work-list variant: bit-sliced
 * variants (1/2-bit data) use nbits bit-plane rows per channel
 * (*rows_per_chan = nbits), the others one packed row per channel. */
int spp_wl_planar_layout(int nbits, int acc, int variant, int64_t nvalid, int32_t omin,
                         int32_t omax, int32_t slot_w, int64_t* halo, int64_t* pitch_w,
                         int64_t* rows_per_chan);
int spp_wl_corner_turn(int nbits, int acc, int variant, const void* in, int bitorder,
                       int64_t nchans, int64_t nsamps, int64_t halo, void* planar,
                       int64_t pitch_w, void* stream);
/* Raw time-major block -> planar rows (channel-major, time packed in words). */
int spp_corner_turn(const void* in, int nbits, int bitorder, int64_t nchans,
                    int64_t nsamps, int64_t halo, void* planar, int64_t pitch_w,
                    void* stream);

/* Self-test of the device-side failure path: launches one CTA whose mbarrier
 * wait can never complete; after limit_ns (<= 1 s) the bounded wait gives up
 * and sets SPP_DEV_TIMEOUT (bit 0) in status[0] (a device status block, as
 * read by spp_status_read).  No trap, no fault: the context stays usable. */
int spp_selftest_wait_timeout(uint32_t* status, uint64_t limit_ns, void* stream);

/* ---- Synthetic inputs (benchmark / test data; no reference counterpart) -------
 * Counter-based generators: element i depends only on (seed, start + i)
 * through the SplitMix64 finaliser, so slices can be regenerated on the host.
 * spp_synth_gauss_u8 maps the upper 32 hash bits through 255 uint32 CDF
 * thresholds (host array); spp_synth_pulse_packed adds +1 (saturating) to the
 * packed field of channel c for rows start_rows[c] .. + width - 1. */
int spp_synth_uniform_bytes(uint8_t* out, int64_t start, int64_t n, uint64_t seed,
                            void* stream);
int spp_synth_gauss_u8(uint8_t* out, int64_t start, int64_t n, uint64_t seed,
                       const uint32_t* thresholds_host, void* stream);
int spp_synth_gauss_f32(float* out, int64_t start, int64_t n, uint64_t seed, float mean,
                        float stdv, void* stream);
int spp_synth_pulse_packed(uint8_t* raw, int64_t nchans, int64_t nsamps, int nbits,
                           int bitorder, const int64_t* start_rows, int width, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SPPGPU_H */
