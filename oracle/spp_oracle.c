/*
 * CPU oracle for the sigpyproc dedispersion path -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatements of the reference algorithms (FRBs/sigpyproc3, paths
 * relative to src/sigpyproc/), used by tests/ to check the CUDA library, by
 * __graft_entry__.smoke() as its checker and by bench.py's CPU-baseline leg.
 * The product never links or calls this file.  Parity of these
 * restatements with the reference's own code is pinned by the golden vectors
 * in tests/golden/ (generated by running the reference numba kernels).
 *
 * Float sums are accumulated in double in channel order (no fast-math), as
 * the reference kernels declare (np.float64 accumulators); the reference's
 * fastmath may reassociate, which is below float32 resolution.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;

void orc_set_threads(int n) { g_threads = n > 0 ? n : 1; }
int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* kernels.unpack{1,2,4}_8_{big,little} (core/kernels.py:20-69): sample k of
 * byte i -> out[i*per + k]; big order puts sample 0 in the high bits. */
void orc_unpack(const uint8_t* in, int64_t nbytes, int nbits, int big, uint8_t* out) {
  const int per = 8 / nbits;
  const unsigned mask = (1u << nbits) - 1u;
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int64_t i = 0; i < nbytes; ++i) {
    const unsigned b = in[i];
    for (int k = 0; k < per; ++k) {
      const int sh = big ? (8 - (k + 1) * nbits) : (k * nbits);
      out[i * per + k] = (uint8_t)((b >> sh) & mask);
    }
  }
}

/* numba array indexing wraps negative indices once (index + size). */
static inline int64_t wrap_neg(int64_t i, int64_t n) { return i < 0 ? i + n : i; }

static int32_t max_abs(const int32_t* d, int64_t n) {
  int32_t m = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t a = d[i] < 0 ? -d[i] : d[i];
    if (a > m) m = a;
  }
  return m;
}

/* kernels.dedisperse (core/kernels.py:340-362), uint8 input:
 *   out[out_start + t] = sum_c in[(t + d_c) * nchans + c], t < nsamps - max|d|,
 * float64 accumulator stored as float32.  Returns the number of outputs. */
int64_t orc_dedisperse_u8(const uint8_t* in, float* out, const int32_t* delays, int64_t nchans,
                          int64_t nsamps, int64_t out_start) {
  const int64_t nvalid = nsamps - max_abs(delays, nchans);
  for (int64_t t = 0; t < nvalid; ++t) {
    double s = 0.0;
    for (int64_t c = 0; c < nchans; ++c) s += in[wrap_neg(t + delays[c], nsamps) * nchans + c];
    out[out_start + t] = (float)s;
  }
  return nvalid > 0 ? nvalid : 0;
}

/* Same for float32 input. */
int64_t orc_dedisperse_f32(const float* in, float* out, const int32_t* delays, int64_t nchans,
                           int64_t nsamps, int64_t out_start) {
  const int64_t nvalid = nsamps - max_abs(delays, nchans);
  for (int64_t t = 0; t < nvalid; ++t) {
    double s = 0.0;
    for (int64_t c = 0; c < nchans; ++c)
      s += (double)in[wrap_neg(t + delays[c], nsamps) * nchans + c];
    out[out_start + t] = (float)s;
  }
  return nvalid > 0 ? nvalid : 0;
}

/* Channel-major copy of a time-major block (cm[c][r] = in[r][c]), so the
 * per-channel loops below read contiguously.  Changes no arithmetic. */
static void *to_channel_major(const void *in, int64_t nchans, int64_t nsamps, size_t esz) {
  void *cm = malloc((size_t)(nchans * nsamps) * esz + 1);
  if (!cm) return NULL;
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int64_t c = 0; c < nchans; ++c) {
    if (esz == 1) {
      const uint8_t *src = (const uint8_t *)in + c;
      uint8_t *dst = (uint8_t *)cm + c * nsamps;
      for (int64_t r = 0; r < nsamps; ++r) dst[r] = src[r * nchans];
    } else {
      const float *src = (const float *)in + c;
      float *dst = (float *)cm + c * nsamps;
      for (int64_t r = 0; r < nsamps; ++r) dst[r] = src[r * nchans];
    }
  }
  return cm;
}

/* DM-trial batch, row-wise R2 contract: out[i][t] = dedisperse(x, D[i])[t]
 * for t < nvalid (= nsamps - max over all |D|), uint8 input, exact int32
 * sums.  Parallel over DM rows. */
void orc_dmt_u8_i32(const uint8_t* in, const int32_t* delays, int64_t ndm, int64_t nchans,
                    int64_t nsamps, int64_t nvalid, int32_t* out, int64_t out_stride) {
  uint8_t *cm = (uint8_t *)to_channel_major(in, nchans, nsamps, 1);
  if (!cm) abort();
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
  for (int64_t i = 0; i < ndm; ++i) {
    const int32_t* d = delays + i * nchans;
    int32_t* o = out + i * out_stride;
    for (int64_t t = 0; t < nvalid; ++t) o[t] = 0;
    for (int64_t c = 0; c < nchans; ++c) {
      const uint8_t* row = cm + c * nsamps;
      const int64_t dc = d[c];
      for (int64_t t = 0; t < nvalid; ++t) o[t] += row[wrap_neg(t + dc, nsamps)];
    }
  }
  free(cm);
}

/* Float32 input: float64 sum per output in channel order, stored float32
 * (and optionally float64 in out64). */
void orc_dmt_f32(const float* in, const int32_t* delays, int64_t ndm, int64_t nchans,
                 int64_t nsamps, int64_t nvalid, float* out, double* out64, int64_t out_stride) {
  float *cm = (float *)to_channel_major(in, nchans, nsamps, 4);
  if (!cm) abort();
#pragma omp parallel num_threads(g_threads)
  {
    double* acc = (double*)malloc(sizeof(double) * (nvalid > 0 ? nvalid : 1));
#pragma omp for schedule(dynamic, 1)
    for (int64_t i = 0; i < ndm; ++i) {
      const int32_t* d = delays + i * nchans;
      for (int64_t t = 0; t < nvalid; ++t) acc[t] = 0.0;
      for (int64_t c = 0; c < nchans; ++c) {
        const float* row = cm + c * nsamps;
        const int64_t dc = d[c];
        for (int64_t t = 0; t < nvalid; ++t) acc[t] += (double)row[wrap_neg(t + dc, nsamps)];
      }
      for (int64_t t = 0; t < nvalid; ++t) {
        if (out) out[i * out_stride + t] = (float)acc[t];
        if (out64) out64[i * out_stride + t] = acc[t];
      }
    }
    free(acc);
  }
  free(cm);
}

/* kernels.dmt_block (core/kernels.py:1155-1168) semantics on time-major
 * input: out[i][t] = sum_c x[(t - d) mod n][c] for t < n (circular roll by
 * +delay, kernels.roll_block :1059-1099), float64 sum, float32 store. */
void orc_dmt_roll_f32(const float* in, const int32_t* delays, int64_t ndm, int64_t nchans,
                      int64_t nsamps, float* out) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
  for (int64_t i = 0; i < ndm; ++i) {
    for (int64_t t = 0; t < nsamps; ++t) {
      double s = 0.0;
      for (int64_t c = 0; c < nchans; ++c) {
        int64_t sh = delays[i * nchans + c] % nsamps;
        if (sh < 0) sh += nsamps;
        int64_t r = t - sh;
        if (r < 0) r += nsamps;
        s += (double)in[r * nchans + c];
      }
      out[i * nsamps + t] = (float)s;
    }
  }
}

/* Packed-input DM batch: unpack (R4) then the row-wise contract, processing
 * DM rows in parallel.  `in` holds nsamps*nchans*nbits/8 bytes. */
void orc_dmt_packed_i32(const uint8_t* in, int nbits, int big, const int32_t* delays, int64_t ndm,
                        int64_t nchans, int64_t nsamps, int64_t nvalid, int32_t* out,
                        int64_t out_stride) {
  const int64_t nbytes = nsamps * nchans * nbits / 8;
  uint8_t* un;
  if (nbits == 8) {
    un = (uint8_t*)in;
  } else {
    un = (uint8_t*)malloc((size_t)(nsamps * nchans));
    orc_unpack(in, nbytes, nbits, big, un);
  }
  orc_dmt_u8_i32(un, delays, ndm, nchans, nsamps, nvalid, out, out_stride);
  if (nbits != 8) free(un);
}

/* kernels.extract_bpass (core/kernels.py:281-292): bpass[c] += x[t][c],
 * float32 accumulation in sample order (bit-exact restatement). */
void orc_bandpass_f32(const float* in, int64_t nchans, int64_t nsamps, float* bpass) {
  for (int64_t t = 0; t < nsamps; ++t)
    for (int64_t c = 0; c < nchans; ++c) bpass[c] = bpass[c] + in[t * nchans + c];
}
void orc_bandpass_u8(const uint8_t* in, int64_t nchans, int64_t nsamps, float* bpass) {
  for (int64_t t = 0; t < nsamps; ++t)
    for (int64_t c = 0; c < nchans; ++c) bpass[c] = bpass[c] + (float)in[t * nchans + c];
}

/* kernels.extract_tim (core/kernels.py:255-278): tim[out_start+t] = sum_c x
 * (float64 accumulator, stored float32). */
void orc_collapse_f32(const float* in, int64_t nchans, int64_t nsamps, float* tim,
                      int64_t out_start) {
  for (int64_t t = 0; t < nsamps; ++t) {
    double s = 0.0;
    for (int64_t c = 0; c < nchans; ++c) s += (double)in[t * nchans + c];
    tim[out_start + t] = (float)s;
  }
}

/* kernels.remove_zerodm (core/kernels.py:465-505), float32 data:
 * y = f32((f64(x) - zdm * f64(w_c)) + f64(b_c)), zdm = sum_c f64(x[t][c]). */
void orc_zero_dm_f32(const float* in, float* out, int64_t nchans, int64_t nsamps,
                     const float* bpass, const float* chanwts) {
#pragma omp parallel for num_threads(g_threads)
  for (int64_t t = 0; t < nsamps; ++t) {
    double z = 0.0;
    for (int64_t c = 0; c < nchans; ++c) z += (double)in[t * nchans + c];
    for (int64_t c = 0; c < nchans; ++c) {
      volatile double t1 = z * (double)chanwts[c];
      volatile double t2 = (double)in[t * nchans + c] - t1;
      out[t * nchans + c] = (float)(t2 + (double)bpass[c]);
    }
  }
}

/* kernels.downsample_1d_mean (core/kernels.py:176-204). */
void orc_downsample_mean(const float* in, int64_t n, int factor, float* out) {
  const int64_t m = n / factor;
  for (int64_t i = 0; i < m; ++i) {
    double s = 0.0;
    for (int k = 0; k < factor; ++k) s += (double)in[i * factor + k];
    out[i] = (float)(s / factor);
  }
}

/* Boxcar matched-filter S/N of one row (TimeSeries.downsample + z-score +
 * apply_boxcar, timeseries.py:107-132, :296-325; core/stats.py:418-477 with
 * loc=mean, scale=std), all in float64:
 *   y = downsample_1d_mean(x, f) (values rounded to float32 as the reference)
 *   snr_w = max_t (sum_{k<w} y[t+k] - w*mean(y)) / (std(y) * sqrt(w)).
 * Writes snr[fi*nwidths + wi] and the argmax t to idx (may be NULL). */
static int cmp_f32(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* numpy's linear-interpolation quantile of sorted float32 values, in float64
 * (numpy _quantile / _lerp: index (n-1)*q, lerp from the far end when the
 * fraction is >= 0.5). */
static double quantile_linear(const float* v, int64_t m, double q) {
  const double vi = (double)(m - 1) * q;
  int64_t lo = (int64_t)floor(vi);
  int64_t hi = lo + 1;
  if (vi >= (double)(m - 1)) lo = hi = m - 1;
  const double g = vi - (double)lo;
  const double a = (double)v[lo], b = (double)v[hi];
  const double diff = b - a;
  return g >= 0.5 ? b - diff * (1.0 - g) : a + diff * g;
}

/* stats.estimate_zscore(loc_method="median", scale_method="iqr")
 * (core/stats.py:418-502) location and scale of float32 values:
 * loc = np.median (float32: mean of the two middle values for an even count),
 * scale = (q75 - q25) / 1.3489795003921634 in float64, replaced by 1 when it
 * is ~0 (np.isclose(scale, 0)). */
void orc_median_iqr(const float* y, int64_t m, double* loc, double* scale) {
  float* v = (float*)malloc(sizeof(float) * (m > 0 ? m : 1));
  memcpy(v, y, sizeof(float) * m);
  qsort(v, (size_t)m, sizeof(float), cmp_f32);
  float med;
  if (m & 1) {
    med = v[(m - 1) / 2];
  } else {
    volatile float sum = v[m / 2 - 1] + v[m / 2];
    med = sum / 2.0f;
  }
  *loc = (double)med;
  double sc = (quantile_linear(v, m, 0.75) - quantile_linear(v, m, 0.25)) / 1.3489795003921634;
  if (fabs(sc) <= 1e-8) sc = 1.0;
  *scale = sc;
  free(v);
}

void orc_boxcar_snr_row_ls(const float* x, int64_t n, const int32_t* factors, int nfactors,
                           const int32_t* widths, int nwidths, int robust, double* snr,
                           int32_t* idx, double* locs, double* scales);

void orc_boxcar_snr_row(const float* x, int64_t n, const int32_t* factors, int nfactors,
                        const int32_t* widths, int nwidths, double* snr, int32_t* idx) {
  orc_boxcar_snr_row_ls(x, n, factors, nfactors, widths, nwidths, 0, snr, idx, NULL, NULL);
}

/* Boxcar S/N of one row per downsample factor and width, with location and
 * scale either mean / population std (robust = 0) or median / IQR (robust =
 * 1):  snr = max_t (sum_{k<w} y[t+k] - w * loc) / (scale * sqrt(w)). */
void orc_boxcar_snr_row_ls(const float* x, int64_t n, const int32_t* factors, int nfactors,
                           const int32_t* widths, int nwidths, int robust, double* snr,
                           int32_t* idx, double* locs, double* scales) {
  float* y = (float*)malloc(sizeof(float) * (n > 0 ? n : 1));
  double* pre = (double*)malloc(sizeof(double) * (n + 1));
  for (int fi = 0; fi < nfactors; ++fi) {
    const int f = factors[fi];
    const int64_t m = n / f;
    orc_downsample_mean(x, n, f, y);
    double s = 0.0, ss = 0.0;
    pre[0] = 0.0;
    for (int64_t i = 0; i < m; ++i) {
      s += (double)y[i];
      pre[i + 1] = s;
    }
    const double mean = m > 0 ? s / (double)m : 0.0;
    for (int64_t i = 0; i < m; ++i) {
      const double dlt = (double)y[i] - mean;
      ss += dlt * dlt;
    }
    double sd = m > 0 ? sqrt(ss / (double)m) : 0.0;
    if (sd == 0.0) sd = 1.0;
    double loc = mean;
    if (robust && m > 0) orc_median_iqr(y, m, &loc, &sd);
    if (locs) locs[fi] = loc;
    if (scales) scales[fi] = sd;
    for (int wi = 0; wi < nwidths; ++wi) {
      const int w = widths[wi];
      double best = -INFINITY;
      int64_t bt = -1;
      for (int64_t t = 0; t + w <= m; ++t) {
        const double v = pre[t + w] - pre[t];
        if (v > best) { best = v; bt = t; }
      }
      snr[fi * nwidths + wi] = bt < 0 ? NAN : (best - (double)w * loc) / (sd * sqrt((double)w));
      if (idx) idx[fi * nwidths + wi] = (int32_t)bt;
    }
  }
  free(y);
  free(pre);
}

/* kernels.subband (core/kernels.py:379-401) with a zero-initialised output:
 * out[t*nsub + chan_to_sub[c]] += in[(t + d_c)*nchans + c], t < nsamps - maxdelay. */
void orc_subband_u8(const uint8_t* in, float* out, const int32_t* delays, const int32_t* chan_to_sub,
                    int64_t maxdelay, int64_t nchans, int64_t nsub, int64_t nsamps) {
  const int64_t nout = nsamps - maxdelay;
  for (int64_t t = 0; t < nout; ++t) {
    for (int64_t s = 0; s < nsub; ++s) out[t * nsub + s] = 0.f;
    for (int64_t c = 0; c < nchans; ++c)
      out[t * nsub + chan_to_sub[c]] += (float)in[wrap_neg(t + delays[c], nsamps) * nchans + c];
  }
}

/* CPU baseline shaped like the reference's parallel path: for each DM row,
 * kernels.dedisperse's loop order (sample outer, channel inner, float64
 * accumulator) on unpacked uint8 samples, rows split across threads the way
 * numba's prange splits work.  Used for the timed CPU baseline only. */
void orc_dmt_rowmajor_u8(const uint8_t* in, const int32_t* delays, int64_t ndm, int64_t nchans,
                         int64_t nsamps, int64_t nvalid, int32_t* out, int64_t out_stride) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(g_threads)
  for (int64_t i = 0; i < ndm; ++i) {
    const int32_t* d = delays + i * nchans;
    for (int64_t t = 0; t < nvalid; ++t) {
      double s = 0.0;
      for (int64_t c = 0; c < nchans; ++c) s += in[wrap_neg(t + d[c], nsamps) * nchans + c];
      out[i * out_stride + t] = (int32_t)s;
    }
  }
}

/* Python's float floor division a // b (CPython float_floor_div: fmod-based,
   so the quotient is the floor of the exact quotient), restated. */
static double py_floordiv(double a, double b) {
  const double mod = fmod(a, b);
  double div = (a - mod) / b;
  if (mod != 0.0 && ((b < 0.0) != (mod < 0.0))) div -= 1.0;
  if (div == 0.0) return copysign(0.0, a / b);
  double fl = floor(div);
  if (div - fl > 0.5) fl += 1.0;
  return fl;
}

/* kernels.fold (core/kernels.py:403-445): one read_plan block into fold_ar /
   count_ar.  The reference takes tsamp, period and accel as float32 and does
   the phase arithmetic in float64, in this order; the bin sums are float32. */
static void orc_fold_impl(const void* in, int is_f32, float* fold_ar, int32_t* count_ar,
                          const int32_t* delays, int32_t maxdelay, float tsamp, float period,
                          float accel, int32_t total_nsamps, int32_t nsamps, int32_t nchans,
                          int32_t nbins, int32_t nints, int32_t nsubs, int32_t index) {
  const double c2 = 2.0 * 299792458.0;
  const double factor1 = (double)total_nsamps / (double)nints;
  const double factor2 = (double)nchans / (double)nsubs;
  const double tobs = (double)total_nsamps * (double)tsamp;
  for (int64_t isamp = 0; isamp < (int64_t)nsamps - maxdelay; ++isamp) {
    const double tj = (double)(isamp + index) * (double)tsamp;
    const double phase =
        (double)nbins * tj * (1.0 + (double)accel * (tj - tobs) / c2) / (double)period + 0.5;
    const int64_t phasebin = llabs((long long)phase) % nbins;
    const double subint = py_floordiv((double)(isamp + index), factor1);
    const double pos1 = subint * nbins * nsubs + (double)phasebin;
    for (int64_t ichan = 0; ichan < nchans; ++ichan) {
      const double sub_band = py_floordiv((double)ichan, factor2);
      const int64_t pos2 = (int64_t)(pos1 + sub_band * nbins);
      int64_t idx = (int64_t)nchans * (isamp + delays[ichan]) + ichan;
      if (idx < 0) idx += (int64_t)nsamps * nchans;  /* numba: negative index wraps */
      const float val = is_f32 ? ((const float*)in)[idx] : (float)((const uint8_t*)in)[idx];
      fold_ar[pos2] = fold_ar[pos2] + val;
      count_ar[pos2] += 1;
    }
  }
}

void orc_fold_block(const void* in, int is_f32, float* fold_ar, int32_t* count_ar,
                    const int32_t* delays, int32_t maxdelay, float tsamp, float period,
                    float accel, int32_t total_nsamps, int32_t nsamps, int32_t nchans,
                    int32_t nbins, int32_t nints, int32_t nsubs, int32_t index) {
  orc_fold_impl(in, is_f32, fold_ar, count_ar, delays, maxdelay, tsamp, period, accel,
                total_nsamps, nsamps, nchans, nbins, nints, nsubs, index);
}

/* The floor division above, exported for its test against Python's own //. */
double orc_py_floordiv(double a, double b) { return py_floordiv(a, b); }
