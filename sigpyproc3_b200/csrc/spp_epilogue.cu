// Channel reductions (bandpass, collapse), zero-DM, downsample, stage-1
// subband, and the boxcar matched-filter S/N epilogue.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>

#include "spp_common.cuh"
#include "spp_dmt.cuh"

namespace spp {

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

// Reads sample (t, c) of a raw time-major block as float (any nbits).
template <int NB>
__device__ __forceinline__ float raw_at(const void* in, int64_t nchans, int64_t t, int64_t c,
                                        int bitorder) {
  if (NB == 32) return static_cast<const float*>(in)[t * nchans + c];
  const uint8_t* b = static_cast<const uint8_t*>(in);
  const int64_t bit = (t * nchans + c) * NB;
  return (float)field_of<NB>(b[bit >> 3], (int)c, bitorder);
}

// ---------------------------------------------------------------------------
// bandpass: per-channel sequential float32 sum over samples, in sample order,
// exactly as kernels.extract_bpass's loop (bit-identical).  One thread per
// channel; 8 samples are loaded ahead of the dependent add chain.
// ---------------------------------------------------------------------------
template <int NB>
__global__ void k_bandpass(const void* __restrict__ in, int64_t nchans, int64_t nsamps,
                           int bitorder, float* __restrict__ bpass) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchans) return;
  float acc = bpass[c];
  int64_t t = 0;
  for (; t + 8 <= nsamps; t += 8) {
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = raw_at<NB>(in, nchans, t + k, c, bitorder);
#pragma unroll
    for (int k = 0; k < 8; ++k) acc = __fadd_rn(acc, v[k]);
  }
  for (; t < nsamps; ++t) acc = __fadd_rn(acc, raw_at<NB>(in, nchans, t, c, bitorder));
  bpass[c] = acc;
}

// collapse: tim[out_start + t] = f32(sum_c f64(x[t][c])) (kernels.extract_tim)
template <int NB>
__global__ void k_collapse(const void* __restrict__ in, int64_t nchans, int64_t nsamps,
                           int bitorder, float* __restrict__ tim, int64_t out_start) {
  const int64_t t = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= nsamps) return;
  double s = 0.0;
  for (int64_t c = lane; c < nchans; c += 32) s += (double)raw_at<NB>(in, nchans, t, c, bitorder);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) tim[out_start + t] = (float)s;
}

// zero-DM on time-major float32 (kernels.remove_zerodm, core/kernels.py:493-505):
// a block of 8 warps takes 256 samples; each warp sums 32 samples' channels in
// channel order (32 x 32 tiles staged through shared memory, one lane per
// sample), then the block rewrites the 256 spectra with coalesced accesses.
// The result is stored in the input's type: float32 rounds; uint8 keeps the low
// eight bits of the truncated value (what the reference's numba cast of a
// float64 to uint8 yields on x86, where values far above 255 are the norm
// because the bandpass is a channel sum).
__device__ __forceinline__ float zdm_store(float, double v) { return (float)v; }
__device__ __forceinline__ uint8_t zdm_store(uint8_t, double v) {
  return (uint8_t)(uint64_t)(int64_t)v;
}

constexpr int kZdmRows = 256;
template <typename T>
__global__ void __launch_bounds__(kZdmRows)
k_zero_dm(const T* __restrict__ in, T* __restrict__ out, int64_t nchans, int64_t nsamps,
          const float* __restrict__ bpass, const float* __restrict__ chanwts) {
  __shared__ float tile[kZdmRows / 32][32][33];
  __shared__ double zs[kZdmRows];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t tb = (int64_t)blockIdx.x * kZdmRows; tb < nsamps; tb += (int64_t)gridDim.x * kZdmRows) {
    const int64_t t0 = tb + warp * 32;
    double s = 0.0;
    for (int64_t c0 = 0; c0 < nchans; c0 += 32) {
      const int64_t c = c0 + lane;
      for (int r = 0; r < 32; ++r) {
        const int64_t t = t0 + r;
        tile[warp][r][lane] = (t < nsamps && c < nchans) ? (float)in[t * nchans + c] : 0.f;
      }
      __syncwarp();
      const int nc = (nchans - c0) < 32 ? (int)(nchans - c0) : 32;
      for (int j = 0; j < nc; ++j) s = __dadd_rn(s, (double)tile[warp][lane][j]);
      __syncwarp();
    }
    zs[threadIdx.x] = s;
    __syncthreads();
    const int64_t rows = imin64(kZdmRows, nsamps - tb);
    for (int64_t r = 0; r < rows; ++r) {
      const double z = zs[r];
      const T* src = in + (tb + r) * nchans;
      T* dst = out + (tb + r) * nchans;
      for (int64_t c = threadIdx.x; c < nchans; c += kZdmRows) {
        const double t1 = __dmul_rn(z, (double)chanwts[c]);
        const double t2 = __dsub_rn((double)src[c], t1);
        dst[c] = zdm_store(T(), __dadd_rn(t2, (double)bpass[c]));
      }
    }
    __syncthreads();
  }
}

// TimeSeries.apply_boxcar (timeseries.py:296-325) over stats.running_filter
// "mean" (core/stats.py:200-243): the series padded symmetrically (np.pad
// "symmetric", a reflection of period 2n), the mean of each window of
// `width` samples times sqrt(width), rolled by ref_bin.  A CTA computes
// kBoxT consecutive window positions i (pre-roll): it stages the padded samples
// they cover in shared memory, each thread sums its first window in float64
// and slides it across kBoxR positions, and writes out[(i + ref_bin) mod n].
constexpr int kBoxThreads = 256;
constexpr int kBoxR = 16;
constexpr int kBoxT = kBoxThreads * kBoxR;

__device__ __forceinline__ int64_t sym_index(int64_t k, int64_t n) {
  int64_t m = k % (2 * n);
  if (m < 0) m += 2 * n;
  return m < n ? m : 2 * n - 1 - m;
}

__global__ void __launch_bounds__(kBoxThreads)
k_boxcar_filter(const float* __restrict__ in, int64_t n, int width, int64_t pad_left,
                int64_t ref_bin, float* __restrict__ out) {
  extern __shared__ float sx[];  // kBoxT + width - 1
  const int64_t i0 = (int64_t)blockIdx.x * kBoxT;
  const int64_t len = imin64(kBoxT, n - i0) + width - 1;
  for (int64_t k = threadIdx.x; k < len; k += kBoxThreads)
    sx[k] = __ldg(in + sym_index(i0 - pad_left + k, n));
  __syncthreads();
  const int64_t a = (int64_t)threadIdx.x * kBoxR;  // this thread's first position
  if (i0 + a >= n) return;
  const int cnt = (int)imin64(kBoxR, n - i0 - a);
  const double norm = sqrt((double)width);
  double s = 0.0;
  for (int k = 0; k < width; ++k) s += (double)sx[a + k];
  for (int r = 0; r < cnt; ++r) {
    if (r > 0) s = (s + (double)sx[a + r + width - 1]) - (double)sx[a + r - 1];
    const int64_t i = i0 + a + r;
    int64_t j = (i + ref_bin) % n;
    if (j < 0) j += n;
    out[j] = (float)(s / (double)width * norm);
  }
}

// downsample_1d_mean over rows
__global__ void k_downsample(const float* __restrict__ in, int64_t n, int64_t in_stride,
                             int factor, float* __restrict__ out, int64_t out_stride) {
  const int64_t m = n / factor;
  const int64_t row = blockIdx.y;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < factor; ++k) s += (double)in[row * in_stride + i * factor + k];
    out[row * out_stride + i] = (float)(s / factor);
  }
}

// downsample_2d_mean_flat
__device__ __forceinline__ float ds_store(float, double v) { return (float)v; }
__device__ __forceinline__ uint8_t ds_store(uint8_t, double v) {
  return (uint8_t)(uint64_t)(int64_t)v;  // numba's float64 -> uint8 cast (truncation)
}

template <typename T>
__global__ void k_downsample_2d(const T* __restrict__ in, int64_t dim1, int64_t dim2,
                                int f1, int f2, T* __restrict__ out) {
  const int64_t n1 = dim1 / f1, n2 = dim2 / f2;
  const int64_t total = n1 * n2;
  const double tot = (double)f1 * f2;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / n2, j = idx - i * n2;
    double s = 0.0;
    const int64_t pos = dim2 * i * f1 + j * f2;
    for (int a = 0; a < f1; ++a)
      for (int b = 0; b < f2; ++b) s += (double)in[pos + a * dim2 + b];
    out[idx] = ds_store(T(), s / tot);
  }
}

// stage-1 subband (kernels.subband with a zeroed output): atomics into
// out[t][sub], exact for integer input (sums < 2^24).
template <int NB>
__global__ void k_subband(const void* __restrict__ in, int64_t nchans, int64_t nsamps,
                          int bitorder, const int32_t* __restrict__ delays,
                          const int32_t* __restrict__ chan_to_sub, int64_t nsub, int64_t nout,
                          float* __restrict__ out) {
  const int64_t total = nout * nchans;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = idx / nchans, c = idx - t * nchans;
    int64_t r = t + delays[c];
    if (r < 0) r += nsamps;
    if (r < 0 || r >= nsamps) continue;
    const int s = chan_to_sub[c];
    if (s < 0 || s >= nsub) continue;
    atomicAdd(out + t * nsub + s, raw_at<NB>(in, nchans, r, c, bitorder));
  }
}

// ---------------------------------------------------------------------------
// Boxcar S/N.  Chunk pass: CTA (chunk k, row r, factor fi) builds the
// downsampled series y over its chunk plus a halo of (wmax-1) samples in
// shared memory as float64, scans it to prefix sums, and records per width the
// best window sum starting inside the chunk (smallest start on ties) plus the
// chunk's sum and second central moment.  Final pass merges chunks (Chan et
// al. 1979 pairwise variance) and forms (best - w*mean) / (std*sqrt(w)).
// ---------------------------------------------------------------------------
constexpr int kSnrChunk = 6144;     // downsampled samples per CTA (24 per thread)
constexpr int kSnrThreads = 256;
constexpr int kSnrMaxW = 4096;
constexpr int kSnrMaxWidths = 32;

struct SnrPart {
  double best;
  int64_t idx;
};

struct SnrCfg {
  int nf, nw, wmax;
  int32_t f[8];
  int32_t w[kSnrMaxWidths];
};

__device__ __forceinline__ double row_val(const void* in, int kind, int64_t i) {
  return kind == SPP_OUT_I32 ? (double)static_cast<const int32_t*>(in)[i]
                             : (double)static_cast<const float*>(in)[i];
}

// One CTA per (chunk of kSnrChunk downsampled samples, row, factor).  Chunk-
// local indices are 32-bit; the width maxima keep per-thread candidates for up
// to kSnrWGroup widths in registers over one pass of the chunk, then reduce
// once (ties go to the smaller sample index, as the reference's argmax).
constexpr int kSnrWGroup = 12;

__global__ void __launch_bounds__(kSnrThreads)
k_snr_chunk(const void* __restrict__ in, int kind, int64_t n, int64_t in_stride, const SnrCfg cfg,
            int64_t nchunks, SnrPart* __restrict__ parts, double* __restrict__ stats) {
  const int nfactors = cfg.nf, nwidths = cfg.nw, wmax = cfg.wmax;
  extern __shared__ double sy[];  // kSnrChunk + wmax + 1
  __shared__ double red_d[kSnrThreads / 32 * kSnrWGroup];
  __shared__ int red_i[kSnrThreads / 32 * kSnrWGroup];
  __shared__ int sw[kSnrMaxWidths];
  __shared__ double carry;
  const int64_t k = blockIdx.x;
  const int64_t row = blockIdx.y / nfactors;
  const int fi = blockIdx.y % nfactors;
  const int f = cfg.f[fi];
  const int64_t m = n / f;
  const int64_t i0 = k * kSnrChunk;
  if (i0 >= m) {
    return;
  }
  const int own = (int)imin64(kSnrChunk, m - i0);
  const int len = (int)imin64(own + wmax, m - i0);  // samples loaded
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < nwidths) sw[threadIdx.x] = cfg.w[threadIdx.x];
  const char* base = static_cast<const char*>(in) + row * in_stride * 4;
  // y values (downsampled means rounded to float32 as the reference output
  // dtype); a power-of-two factor divides exactly by multiplying
  const bool pow2 = (f & (f - 1)) == 0;
  const double inv = 1.0 / (double)f;
  for (int j = threadIdx.x; j < len; j += blockDim.x) {
    double s = 0.0;
    const int64_t x0 = (i0 + j) * f;
    for (int q = 0; q < f; ++q) s += row_val(base, kind, x0 + q);
    sy[j + 1] = (double)(float)(pow2 ? s * inv : s / f);
  }
  if (threadIdx.x == 0) { sy[0] = 0.0; carry = 0.0; }
  __syncthreads();
  // chunk sum and M2 over owned samples
  {
    double s = 0.0;
    for (int j = threadIdx.x; j < own; j += blockDim.x) s += sy[j + 1];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red_d[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kSnrThreads / 32; ++w) t += red_d[w];
      carry = t;
    }
    __syncthreads();
    const double mu = carry / (double)own;
    double q = 0.0;
    for (int j = threadIdx.x; j < own; j += blockDim.x) {
      const double d = sy[j + 1] - mu;
      q += d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    __syncthreads();
    if (lane == 0) red_d[warp] = q;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kSnrThreads / 32; ++w) t += red_d[w];
      double* st = stats + ((row * nfactors + fi) * nchunks + k) * 3;
      st[0] = (double)own;
      st[1] = carry;
      st[2] = t;
    }
    __syncthreads();
  }
  // inclusive scan of sy[1..len] (sequential per thread segment + warp/block scan)
  {
    const int per = (len + blockDim.x - 1) / blockDim.x;
    const int a = 1 + threadIdx.x * per;
    const int b = min(a + per, len + 1);
    double s = 0.0;
    for (int j = a; j < b; ++j) { s += sy[j]; sy[j] = s; }
    double incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) red_d[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      double acc = 0.0;
      for (int w = 0; w < kSnrThreads / 32; ++w) { const double v = red_d[w]; red_d[w] = acc; acc += v; }
    }
    __syncthreads();
    const double off = red_d[warp] + (incl - s);
    for (int j = a; j < b; ++j) sy[j] += off;
    __syncthreads();
  }
  // window maxima: widths in groups of kSnrWGroup, one pass over the chunk each
  for (int w0 = 0; w0 < nwidths; w0 += kSnrWGroup) {
    double best[kSnrWGroup];
    int bt[kSnrWGroup], wv[kSnrWGroup];
#pragma unroll
    for (int g = 0; g < kSnrWGroup; ++g) {
      best[g] = -DBL_MAX;
      bt[g] = INT_MAX;
      wv[g] = (w0 + g < nwidths) ? sw[w0 + g] : INT_MAX / 2;
    }
    const int ng = min(kSnrWGroup, nwidths - w0);
    if (len == own + wmax) {
      // interior chunk: every window of every owned sample is loaded
      for (int t = threadIdx.x; t < own; t += blockDim.x) {
        const double p0 = sy[t];
#pragma unroll
        for (int g = 0; g < kSnrWGroup; ++g) {
          if (g < ng) {
            const double v = sy[t + wv[g]] - p0;
            if (v > best[g]) { best[g] = v; bt[g] = t; }
          }
        }
      }
    } else {
      for (int t = threadIdx.x; t < own; t += blockDim.x) {
        const double p0 = sy[t];
#pragma unroll
        for (int g = 0; g < kSnrWGroup; ++g) {
          if (t + wv[g] <= len) {  // window inside the row
            const double v = sy[t + wv[g]] - p0;
            if (v > best[g]) { best[g] = v; bt[g] = t; }
          }
        }
      }
    }
#pragma unroll
    for (int g = 0; g < kSnrWGroup; ++g) {
      if (g >= ng) break;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best[g], o);
        const int oi = __shfl_xor_sync(0xffffffffu, bt[g], o);
        if (ov > best[g] || (ov == best[g] && oi < bt[g])) { best[g] = ov; bt[g] = oi; }
      }
      if (lane == 0) { red_d[warp * kSnrWGroup + g] = best[g]; red_i[warp * kSnrWGroup + g] = bt[g]; }
    }
    __syncthreads();
    if (threadIdx.x < kSnrWGroup && w0 + (int)threadIdx.x < nwidths) {
      const int g = threadIdx.x;
      double bb = red_d[g];
      int bi = red_i[g];
      for (int w2 = 1; w2 < kSnrThreads / 32; ++w2) {
        const double v = red_d[w2 * kSnrWGroup + g];
        const int vi = red_i[w2 * kSnrWGroup + g];
        if (v > bb || (v == bb && vi < bi)) { bb = v; bi = vi; }
      }
      SnrPart* p = parts + (((row * nfactors + fi) * nwidths + (w0 + g)) * nchunks + k);
      p->best = bb;
      p->idx = bi == INT_MAX ? LLONG_MAX : i0 + bi;
    }
    __syncthreads();
  }
}

__global__ void k_snr_final(int64_t n, const SnrCfg cfg, int64_t nrows, int64_t nchunks, const SnrPart* __restrict__ parts,
                            const double* __restrict__ stats, float* __restrict__ snr,
                            int32_t* __restrict__ peak, const double* __restrict__ locscale) {
  const int nfactors = cfg.nf, nwidths = cfg.nw;
  const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nrows * nfactors * nwidths) return;
  const int wi = id % nwidths;
  const int64_t rf = id / nwidths;  // row * nfactors + fi
  const int fi = rf % nfactors;
  const int64_t m = n / cfg.f[fi];
  const int64_t nck = (m + kSnrChunk - 1) / kSnrChunk;
  // merge moments
  double cnt = 0.0, mean = 0.0, m2 = 0.0;
  for (int64_t k = 0; k < nck; ++k) {
    const double* st = stats + (rf * nchunks + k) * 3;
    const double nb = st[0];
    if (nb <= 0) continue;
    const double mb = st[1] / nb;
    const double d = mb - mean;
    const double tot = cnt + nb;
    mean += d * nb / tot;
    m2 += st[2] + d * d * cnt * nb / tot;
    cnt = tot;
  }
  double sd = cnt > 0 ? sqrt(m2 / cnt) : 0.0;
  if (sd == 0.0) sd = 1.0;
  if (locscale) {  // median / IQR scale computed by k_row_quantiles
    mean = locscale[rf * 2];
    sd = locscale[rf * 2 + 1];
  }
  double best = -DBL_MAX;
  long long bidx = -1;
  for (int64_t k = 0; k < nck; ++k) {
    const SnrPart p = parts[(rf * nwidths + wi) * nchunks + k];
    if (p.idx < 0 || p.idx == LLONG_MAX) continue;
    if (p.best > best) { best = p.best; bidx = p.idx; }
  }
  const int w = cfg.w[wi];
  snr[id] = bidx < 0 ? NAN : (float)((best - (double)w * mean) / (sd * sqrt((double)w)));
  if (peak) peak[id] = (int32_t)bidx;
}

// ---------------------------------------------------------------------------
// Median / IQR of each downsampled row (the S/N epilogue's robust z-score:
// stats.estimate_zscore with loc "median" and scale "iqr", core/stats.py:
// 418-502).  One CTA per (row, factor): the y values (the same float32
// downsampled means as k_snr_chunk) are mapped to order-preserving 32-bit keys
// and the needed order statistics are found exactly by radix selection, three
// passes of 11/11/10-bit digits with one shared-memory histogram per distinct
// key prefix (warp-aggregated increments).  Up to six ranks: the two middle
// values (median) and the two neighbours of each quartile's index (q25, q75,
// linear interpolation as numpy's percentile).
// ---------------------------------------------------------------------------
constexpr int kQThreads = 256;
constexpr int kQBits = 11;
constexpr int kQBins = 1 << kQBits;
constexpr int kQRanks = 6;

__device__ __forceinline__ uint32_t f32_key(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ float key_f32(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ __forceinline__ float snr_y(const char* base, int kind, int64_t i, int f, bool pow2,
                                       double inv) {
  double s = 0.0;
  const int64_t x0 = i * f;
  for (int q = 0; q < f; ++q) s += row_val(base, kind, x0 + q);
  return (float)(pow2 ? s * inv : s / f);
}

__device__ __forceinline__ double quantile_lerp(double a, double b, double g) {
  const double diff = b - a;  // numpy _lerp: from the far end when g >= 0.5
  return g >= 0.5 ? b - diff * (1.0 - g) : a + diff * g;
}

__global__ void __launch_bounds__(kQThreads)
k_row_quantiles(const void* __restrict__ in, int kind, int64_t n, int64_t in_stride,
                const SnrCfg cfg, double* __restrict__ locscale) {
  extern __shared__ uint32_t qhist[];  // kQRanks x kQBins
  __shared__ uint32_t pre[kQRanks];    // key prefix per rank (bits above the digit)
  __shared__ int64_t rnk[kQRanks];     // rank within the prefix
  __shared__ uint32_t dpre[kQRanks];   // distinct prefixes this pass
  __shared__ int slot[kQRanks];        // rank -> distinct-prefix histogram
  __shared__ int ndist;
  const int64_t row = blockIdx.x / cfg.nf;
  const int fi = blockIdx.x % cfg.nf;
  const int f = cfg.f[fi];
  const int64_t m = n / f;
  const char* base = static_cast<const char*>(in) + row * in_stride * 4;
  const bool pow2 = (f & (f - 1)) == 0;
  const double inv = 1.0 / (double)f;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // ranks: median pair, then q25 and q75 neighbours (0-based, in [0, m))
  const double v25 = (double)(m - 1) * 0.25, v75 = (double)(m - 1) * 0.75;
  const int64_t l25 = (int64_t)floor(v25), l75 = (int64_t)floor(v75);
  if (threadIdx.x == 0) {
    const int64_t r[kQRanks] = {(m - 1) / 2, m / 2, l25, l25 + 1 < m ? l25 + 1 : m - 1,
                                l75, l75 + 1 < m ? l75 + 1 : m - 1};
    for (int t = 0; t < kQRanks; ++t) { pre[t] = 0u; rnk[t] = r[t]; }
  }
  __syncthreads();
  const int shifts[3] = {21, 10, 0};
  const int widths[3] = {11, 11, 10};
  for (int pass = 0; pass < 3; ++pass) {
    const int sh = shifts[pass], wb = widths[pass];
    const uint32_t hi_mask = (sh + wb >= 32) ? 0u : ~((1u << (sh + wb)) - 1u);
    const uint32_t dmask = (1u << wb) - 1u;
    if (threadIdx.x == 0) {
      int nd = 0;
      for (int t = 0; t < kQRanks; ++t) {
        int k = 0;
        while (k < nd && dpre[k] != pre[t]) ++k;
        if (k == nd) dpre[nd++] = pre[t];
        slot[t] = k;
      }
      ndist = nd;
    }
    for (int i = threadIdx.x; i < kQRanks * kQBins; i += kQThreads) qhist[i] = 0u;
    __syncthreads();
    const int nd = ndist;
    const int64_t mr = (m + kQThreads - 1) / kQThreads * kQThreads;  // whole warps iterate
    for (int64_t i = threadIdx.x; i < mr; i += kQThreads) {
      int id = -1;
      if (i < m) {
        const uint32_t key = f32_key(snr_y(base, kind, i, f, pow2, inv));
        const uint32_t hp = key & hi_mask;
        for (int k = 0; k < nd; ++k)
          if (dpre[k] == hp) { id = k * kQBins + (int)((key >> sh) & dmask); break; }
      }
      const unsigned peers = __match_any_sync(0xffffffffu, id);
      if (id >= 0 && lane == __ffs(peers) - 1) atomicAdd(&qhist[id], (uint32_t)__popc(peers));
    }
    __syncthreads();
    // one warp per rank: the digit whose cumulative count passes the rank
    if (warp < kQRanks) {
      const uint32_t* h = qhist + slot[warp] * kQBins;
      constexpr int per = kQBins / 32;
      uint32_t sum = 0;
      for (int j = 0; j < per; ++j) sum += h[lane * per + j];
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int64_t r = rnk[warp];
      const uint32_t excl = incl - sum;
      const unsigned hit = __ballot_sync(0xffffffffu, (int64_t)excl <= r && r < (int64_t)incl);
      const int src = __ffs(hit) - 1;
      if (lane == src) {
        int64_t c = excl;
        int d = lane * per;
        for (int j = 0; j < per; ++j, ++d) {
          if (r < c + (int64_t)h[d]) break;
          c += h[d];
        }
        rnk[warp] = r - c;
        pre[warp] |= (uint32_t)d << sh;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    float med;
    if (m & 1) {
      med = key_f32(pre[0]);
    } else {
      med = __fmul_rn(__fadd_rn(key_f32(pre[0]), key_f32(pre[1])), 0.5f);
    }
    const double q25 = quantile_lerp((double)key_f32(pre[2]), (double)key_f32(pre[3]),
                                     v25 - (double)l25);
    const double q75 = quantile_lerp((double)key_f32(pre[4]), (double)key_f32(pre[5]),
                                     v75 - (double)l75);
    double sc = (q75 - q25) / 1.3489795003921634;
    if (fabs(sc) <= 1e-8) sc = 1.0;  // np.isclose(scale, 0) -> 1
    locscale[blockIdx.x * 2] = (double)med;
    locscale[blockIdx.x * 2 + 1] = sc;
  }
}

// ---------------------------------------------------------------------------
// MatchedFilter (core/filters.py:29-338, kernels.convolve_templates
// core/kernels.py:861-906): the reference correlates the z-scored series with
// each template by FFT over the series repeated to the FFT length N >= n
// (circular_pad_goodsize), the template zero-padded to N, its reference bin
// moved to index 0, time-reversed and normalised to zero mean and unit power
// over all N entries.  That is, for t < n,
//   conv[t] = (sum_j h[j] * z[((t + j - ref) mod N) mod n] - mu * S) / sigma,
// mu = sum(h) / N, sigma = sqrt(sum(h^2) - sum(h)^2 / N), S = sum_{m<N} z[m mod n],
// computed here directly in float64 (the templates are at most a few hundred
// bins) and stored float32 as the reference's convs.
// ---------------------------------------------------------------------------
__global__ void k_zscore(const float* __restrict__ in, int64_t n, const double* __restrict__ ls,
                         float* __restrict__ out) {
  // np.subtract(x, loc, dtype=float32) then np.divide(., scale) into float32
  const float loc = (float)ls[0];
  const double scale = ls[1];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)((double)__fsub_rn(in[i], loc) / scale);
}

// mean and population standard deviation of one row in float64 (loc/scale
// "mean"/"std"), one CTA per row
__global__ void k_row_mean_std(const void* __restrict__ in, int kind, int64_t n, int64_t in_stride,
                               double* __restrict__ ls) {
  __shared__ double red[32];
  const char* base = static_cast<const char*>(in) + (int64_t)blockIdx.x * in_stride * 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += row_val(base, kind, i);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w];
    red[31] = t / (double)n;
  }
  __syncthreads();
  const double mean = red[31];
  __syncthreads();
  double q = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double d = row_val(base, kind, i) - mean;
    q += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
  if (lane == 0) red[warp] = q;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w];
    double sd = sqrt(t / (double)n);
    if (fabs(sd) <= 1e-8) sd = 1.0;  // np.isclose(scale, 0) -> 1
    ls[blockIdx.x * 2] = mean;
    ls[blockIdx.x * 2 + 1] = sd;
  }
}

// S = sum_{m < N} z[m mod n] in float64, one CTA
__global__ void k_padded_sum(const float* __restrict__ z, int64_t n, int64_t nfft,
                             double* __restrict__ out) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int64_t reps = nfft / n, rem = nfft % n;
  double full = 0.0, part = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = (double)z[i];
    full += v;
    if (i < rem) part += v;
  }
  double t = full * (double)reps + part;
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) red[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int w = 0; w < nw; ++w) u += red[w];
    out[0] = u;
  }
}

// First maximum of convs in flattened (template, sample) order, as np.argmax:
// the float's order-preserving key in the high word and the complement of the
// flat index in the low word, so atomicMax keeps the largest value and, among
// equal values, the smallest index.
__global__ void k_argmax_first(const float* __restrict__ v, int64_t count,
                               unsigned long long* __restrict__ best) {
  __shared__ unsigned long long red[32];
  unsigned long long b = 0ull;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long key =
        ((unsigned long long)f32_key(v[i]) << 32) | (unsigned long long)(0xFFFFFFFFu - (uint32_t)i);
    if (key > b) b = key;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(0xffffffffu, b, o);
    if (ob > b) b = ob;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (red[w] > b) b = red[w];
    b = red[0] > b ? red[0] : b;
    atomicMax(best, b);
  }
}

// conv[k][t]: one thread per output sample of one template (blockIdx.y)
__global__ void k_template_conv(const float* __restrict__ z, int64_t n, int64_t nfft,
                                const double* __restrict__ temps, const int32_t* __restrict__ toff,
                                const int32_t* __restrict__ tref, const double* __restrict__ tstat,
                                const double* __restrict__ spad, float* __restrict__ convs) {
  const int k = blockIdx.y;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double* h = temps + toff[k];
  const int len = toff[k + 1] - toff[k];
  const int64_t ref = tref[k];
  double acc = 0.0;
  int64_t m = t - ref;  // padded index of h[0], taken mod N then mod n
  m %= nfft;
  if (m < 0) m += nfft;
  for (int j = 0; j < len; ++j) {
    acc += h[j] * (double)z[m % n];
    if (++m == nfft) m = 0;
  }
  // tstat[k]: (mu, sigma) of the padded, normalised template
  const double mu = tstat[2 * k], sigma = tstat[2 * k + 1];
  convs[(int64_t)k * n + t] = (float)(sigma > 0.0 ? (acc - mu * spad[0]) / sigma : acc - mu * spad[0]);
}

template <typename F>
static int dispatch_nb(int nbits, F&& f) {
  switch (nbits) {
    case 1: f(std::integral_constant<int, 1>()); return SPP_OK;
    case 2: f(std::integral_constant<int, 2>()); return SPP_OK;
    case 4: f(std::integral_constant<int, 4>()); return SPP_OK;
    case 8: f(std::integral_constant<int, 8>()); return SPP_OK;
    case 32: f(std::integral_constant<int, 32>()); return SPP_OK;
    default: return fail(SPP_ERR_ARG, "nbits must be 1, 2, 4, 8 or 32 (got %d)", nbits);
  }
}

static int check_raw(const void* in, int nbits, int bitorder, int64_t nchans, int64_t nsamps) {
  if (!in) return fail(SPP_ERR_ARG, "null input");
  if (nchans <= 0 || nsamps < 0) return fail(SPP_ERR_ARG, "bad shape");
  if (nbits < 8 && (nchans * nbits) % 8) return fail(SPP_ERR_ARG, "nchans*nbits must be a multiple of 8");
  if (bitorder != SPP_BITORDER_BIG && bitorder != SPP_BITORDER_LITTLE) return fail(SPP_ERR_ARG, "bad bitorder");
  return SPP_OK;
}

}  // namespace spp

using namespace spp;

extern "C" {

int spp_bandpass(const void* in, int nbits, int bitorder, int64_t nchans, int64_t nsamps,
                 float* bpass, void* stream) {
  int rc = check_raw(in, nbits, bitorder, nchans, nsamps);
  if (rc) return rc;
  if (!bpass) return fail(SPP_ERR_ARG, "null bpass");
  if (nsamps == 0) return SPP_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned blocks = (unsigned)ceil_div(nchans, 128);
  rc = dispatch_nb(nbits, [&](auto nb) {
    k_bandpass<decltype(nb)::value><<<blocks, 128, 0, st>>>(in, nchans, nsamps, bitorder, bpass);
  });
  if (rc) return rc;
  return cuda_status(cudaGetLastError(), "bandpass launch");
}

int spp_collapse(const void* in, int nbits, int bitorder, int64_t nchans, int64_t nsamps,
                 float* tim, int64_t out_start, void* stream) {
  int rc = check_raw(in, nbits, bitorder, nchans, nsamps);
  if (rc) return rc;
  if (!tim || out_start < 0) return fail(SPP_ERR_ARG, "bad output");
  if (nsamps == 0) return SPP_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned blocks = (unsigned)ceil_div(nsamps, 8);
  rc = dispatch_nb(nbits, [&](auto nb) {
    k_collapse<decltype(nb)::value><<<blocks, 256, 0, st>>>(in, nchans, nsamps, bitorder, tim, out_start);
  });
  if (rc) return rc;
  return cuda_status(cudaGetLastError(), "collapse launch");
}

int spp_zero_dm(const float* in, float* out, int64_t nchans, int64_t nsamps, const float* bpass,
                const float* chanwts, void* stream) {
  if (!in || !out || !bpass || !chanwts) return fail(SPP_ERR_ARG, "null pointer");
  if (nchans <= 0 || nsamps < 0) return fail(SPP_ERR_ARG, "bad shape");
  if (nsamps == 0) return SPP_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(nsamps, kZdmRows), 148 * 6);
  k_zero_dm<float><<<blocks, kZdmRows, 0, as_stream(stream)>>>(in, out, nchans, nsamps, bpass,
                                                               chanwts);
  return cuda_status(cudaGetLastError(), "zero_dm launch");
}

int spp_zero_dm_u8(const uint8_t* in, uint8_t* out, int64_t nchans, int64_t nsamps,
                   const float* bpass, const float* chanwts, void* stream) {
  if (!in || !out || !bpass || !chanwts) return fail(SPP_ERR_ARG, "null pointer");
  if (nchans <= 0 || nsamps < 0) return fail(SPP_ERR_ARG, "bad shape");
  if (nsamps == 0) return SPP_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(nsamps, kZdmRows), 148 * 6);
  k_zero_dm<uint8_t><<<blocks, kZdmRows, 0, as_stream(stream)>>>(in, out, nchans, nsamps, bpass,
                                                                 chanwts);
  return cuda_status(cudaGetLastError(), "zero_dm launch");
}

int spp_downsample_mean(const float* in, int64_t nrows, int64_t n, int64_t in_stride, int factor,
                        float* out, int64_t out_stride, void* stream) {
  if (!in || !out) return fail(SPP_ERR_ARG, "null pointer");
  if (factor <= 0) return fail(SPP_ERR_ARG, "Factor must be a positive integer.");
  if (nrows <= 0 || n < 0) return fail(SPP_ERR_ARG, "bad shape");
  if (factor > n) return fail(SPP_ERR_ARG, "Factor must be less than the size of the array.");
  if (nrows > 65535) return fail(SPP_ERR_UNSUPPORTED, "too many rows");
  const int64_t m = n / factor;
  dim3 grid((unsigned)std::min<int64_t>(ceil_div(m, 256), 4096), (unsigned)nrows);
  k_downsample<<<grid, 256, 0, as_stream(stream)>>>(in, n, in_stride, factor, out, out_stride);
  return cuda_status(cudaGetLastError(), "downsample launch");
}

int spp_downsample_2d_mean(const float* in, int64_t dim1, int64_t dim2, int factor1, int factor2,
                           float* out, void* stream) {
  if (!in || !out) return fail(SPP_ERR_ARG, "null pointer");
  if (factor1 <= 0 || factor2 <= 0) return fail(SPP_ERR_ARG, "factors must be positive");
  const int64_t total = (dim1 / factor1) * (dim2 / factor2);
  if (total == 0) return SPP_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(total, 256), 148 * 32);
  k_downsample_2d<float><<<blocks, 256, 0, as_stream(stream)>>>(in, dim1, dim2, factor1, factor2, out);
  return cuda_status(cudaGetLastError(), "downsample_2d launch");
}

int spp_downsample_2d_mean_u8(const uint8_t* in, int64_t dim1, int64_t dim2, int factor1,
                              int factor2, uint8_t* out, void* stream) {
  if (!in || !out) return fail(SPP_ERR_ARG, "null pointer");
  if (factor1 <= 0 || factor2 <= 0 || dim1 < 0 || dim2 < 0) return fail(SPP_ERR_ARG, "bad factors");
  const int64_t total = (dim1 / factor1) * (dim2 / factor2);
  if (total == 0) return SPP_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(total, 256), 148 * 32);
  k_downsample_2d<uint8_t><<<blocks, 256, 0, as_stream(stream)>>>(in, dim1, dim2, factor1, factor2,
                                                                  out);
  return cuda_status(cudaGetLastError(), "downsample_2d launch");
}

int spp_subband(const void* in, int nbits, int bitorder, int64_t nchans, int64_t nsamps,
                const int32_t* delays, int32_t maxdelay, const int32_t* chan_to_sub, int64_t nsub,
                float* out, void* stream) {
  int rc = check_raw(in, nbits, bitorder, nchans, nsamps);
  if (rc) return rc;
  if (!delays || !chan_to_sub || !out || nsub <= 0) return fail(SPP_ERR_ARG, "bad arguments");
  const int64_t nout = nsamps - maxdelay;
  if (nout <= 0) return SPP_OK;
  cudaStream_t st = as_stream(stream);
  rc = cuda_status(cudaMemsetAsync(out, 0, sizeof(float) * nout * nsub, st), "subband memset");
  if (rc) return rc;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(nout * nchans, 256), 148 * 64);
  rc = dispatch_nb(nbits, [&](auto nb) {
    k_subband<decltype(nb)::value><<<blocks, 256, 0, st>>>(in, nchans, nsamps, bitorder, delays,
                                                           chan_to_sub, nsub, nout, out);
  });
  if (rc) return rc;
  return cuda_status(cudaGetLastError(), "subband launch");
}

}  // extern "C"

// Sizes the S/N workspace for `n` samples per row.
int64_t snr_ws(int64_t nrows, int64_t n, int nfactors, int nwidths, int64_t* nchunks) {
  const int64_t nck = ceil_div(std::max<int64_t>(n, 1), kSnrChunk);
  *nchunks = nck;
  const int64_t parts = nrows * nfactors * nwidths * nck * (int64_t)sizeof(SnrPart);
  const int64_t stats = nrows * nfactors * nck * 3 * (int64_t)sizeof(double);
  return kStatusBytes + round_up(parts, 256) + round_up(stats, 256);
}

extern "C" {

int64_t spp_boxcar_snr_workspace_bytes(int64_t nrows, int64_t n, int nfactors, int nwidths) {
  int64_t nck;
  return snr_ws(nrows, n, nfactors, nwidths, &nck);
}

}  // extern "C"

static int boxcar_snr_impl(const void* in, int in_kind, int64_t nrows, int64_t n,
                           int64_t in_stride, const int32_t* factors, int nfactors,
                           const int32_t* widths, int nwidths, float* snr, int32_t* peak_index,
                           void* workspace, int64_t workspace_bytes, void* stream, bool robust) {
  if (!in || !factors || !widths || !snr || !workspace) return fail(SPP_ERR_ARG, "null pointer");
  if (in_kind != SPP_OUT_F32 && in_kind != SPP_OUT_I32) return fail(SPP_ERR_ARG, "bad in_kind");
  if (nrows <= 0 || n <= 0 || nfactors <= 0 || nfactors > 8 || nwidths <= 0 ||
      nwidths > kSnrMaxWidths)
    return fail(SPP_ERR_ARG, "bad sizes (nfactors <= 8, nwidths <= %d)", kSnrMaxWidths);
  if (nrows * nfactors > 65535) return fail(SPP_ERR_UNSUPPORTED, "rows*factors > 65535");
  SnrCfg cfg{};
  cfg.nf = nfactors;
  cfg.nw = nwidths;
  cfg.wmax = 1;
  for (int i = 0; i < nfactors; ++i) {
    if (factors[i] <= 0 || factors[i] > n) return fail(SPP_ERR_ARG, "invalid downsample factor %d", factors[i]);
    cfg.f[i] = factors[i];
  }
  for (int i = 0; i < nwidths; ++i) {
    if (widths[i] < 1 || widths[i] > kSnrMaxW) return fail(SPP_ERR_ARG, "invalid boxcar width: %d", widths[i]);
    cfg.w[i] = widths[i];
    cfg.wmax = std::max(cfg.wmax, (int)widths[i]);
  }
  int64_t nck;
  const int64_t base_need = snr_ws(nrows, n, nfactors, nwidths, &nck);
  const int64_t need = base_need + (robust ? round_up(nrows * nfactors * 16, 256) : 0);
  if (workspace_bytes < need)
    return fail(SPP_ERR_SIZE, "workspace %lld < %lld", (long long)workspace_bytes, (long long)need);
  cudaStream_t st = as_stream(stream);
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  SnrPart* parts = reinterpret_cast<SnrPart*>(ws + kStatusBytes);
  double* stats = reinterpret_cast<double*>(
      ws + kStatusBytes + round_up(nrows * nfactors * nwidths * nck * (int64_t)sizeof(SnrPart), 256));
  int rc = cuda_status(cudaMemsetAsync(parts, 0xFF, sizeof(SnrPart) * nrows * nfactors * nwidths * nck, st), "parts init");
  if (rc) return rc;
  rc = cuda_status(cudaMemsetAsync(stats, 0, sizeof(double) * 3 * nrows * nfactors * nck, st), "stats init");
  if (rc) return rc;
  const int64_t smem = (int64_t)(kSnrChunk + cfg.wmax + 1) * 8;
  if (smem > 48 * 1024) {
    rc = set_smem_attr(reinterpret_cast<const void*>(k_snr_chunk), smem);
    if (rc) return rc;
  }
  dim3 grid((unsigned)nck, (unsigned)(nrows * nfactors));
  k_snr_chunk<<<grid, kSnrThreads, smem, st>>>(in, in_kind, n, in_stride, cfg, nck, parts, stats);
  rc = cuda_status(cudaGetLastError(), "snr chunk launch");
  if (rc) return rc;
  double* locscale = nullptr;
  if (robust) {
    locscale = reinterpret_cast<double*>(ws + base_need);
    const int64_t qsmem = (int64_t)kQRanks * kQBins * 4;
    rc = set_smem_attr(reinterpret_cast<const void*>(k_row_quantiles), qsmem);
    if (rc) return rc;
    k_row_quantiles<<<(unsigned)(nrows * nfactors), kQThreads, qsmem, st>>>(in, in_kind, n,
                                                                          in_stride, cfg, locscale);
    rc = cuda_status(cudaGetLastError(), "row quantiles launch");
    if (rc) return rc;
  }
  const int64_t nout = nrows * nfactors * nwidths;
  k_snr_final<<<(unsigned)ceil_div(nout, 256), 256, 0, st>>>(n, cfg, nrows, nck, parts, stats, snr,
                                                             peak_index, locscale);
  return cuda_status(cudaGetLastError(), "snr final launch");
}

// ---------------------------------------------------------------------------
// Median absolute deviation of each row (stats._scale_mad, core/stats.py:
// 505-536, with estimate_loc's float32 median, core/stats.py:284-326).  One
// CTA per row: the two middle values by radix selection over order-preserving
// 32-bit float keys give the float32 median (averaged in float32) and the
// float64 one (averaged in float64, as np.median of the float64 copy); the
// two middle absolute deviations |f64(x) - median64| by radix selection over
// their 64-bit patterns (non-negative doubles order as unsigned integers) give
// the MAD, divided by Phi^-1(3/4); a MAD within 1e-8 of 0 is replaced by the
// mean absolute deviation over sqrt(2/pi) (a float64 sum in another order
// than numpy's pairwise one), and a scale within 1e-8 of 0 by 1.
// ---------------------------------------------------------------------------

// Ranks r0 <= r1 of n keys by radix selection in one CTA: digits of kQBits
// from the top; each pass histograms (warp-aggregated shared atomics) the
// keys that match a rank's fixed higher digits, then fixes that rank's next
// digit.  `out` (shared) receives the two keys.
template <typename K, class KeyF>
__device__ void select_pair(int64_t n, int64_t r0, int64_t r1, const KeyF& key, uint32_t* hist,
                            K* out) {
  constexpr int kBits = (int)sizeof(K) * 8;
  __shared__ K pre[2];
  __shared__ long long rk[2];
  if (threadIdx.x == 0) {
    pre[0] = pre[1] = K(0);
    rk[0] = r0;
    rk[1] = r1;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int hi = kBits; hi > 0; hi -= kQBits) {
    const int lo = hi > kQBits ? hi - kQBits : 0;
    const int wb = hi - lo;
    const K himask = hi >= kBits ? K(0) : ~((K(1) << hi) - K(1));
    const K dmask = (K(1) << wb) - K(1);
    for (int i = threadIdx.x; i < 2 * kQBins; i += blockDim.x) hist[i] = 0u;
    __syncthreads();
    const K p0 = pre[0], p1 = pre[1];
    const int64_t nr = (n + blockDim.x - 1) / blockDim.x * blockDim.x;  // whole warps iterate
    for (int64_t i = threadIdx.x; i < nr; i += blockDim.x) {
      int id0 = -1, id1 = -1;
      if (i < n) {
        const K k = key(i);
        const int dig = (int)((k >> lo) & dmask);
        if ((k & himask) == p0) id0 = dig;
        if ((k & himask) == p1) id1 = kQBins + dig;
      }
      unsigned peers = __match_any_sync(0xffffffffu, id0);
      if (id0 >= 0 && lane == __ffs(peers) - 1) atomicAdd(&hist[id0], (uint32_t)__popc(peers));
      peers = __match_any_sync(0xffffffffu, id1);
      if (id1 >= 0 && lane == __ffs(peers) - 1) atomicAdd(&hist[id1], (uint32_t)__popc(peers));
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      const int r = threadIdx.x;
      const uint32_t* h = hist + r * kQBins;
      long long c = 0;
      int d = 0;
      for (; d < (1 << wb) - 1; ++d) {
        if (rk[r] < c + (long long)h[d]) break;
        c += h[d];
      }
      rk[r] -= c;
      pre[r] |= K(d) << lo;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = pre[0];
    out[1] = pre[1];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kQThreads)
k_row_mad(const void* __restrict__ in, int kind, int64_t n, int64_t in_stride,
          double* __restrict__ locscale) {
  __shared__ uint32_t hist[2 * kQBins];
  __shared__ uint32_t k32[2];
  __shared__ unsigned long long k64[2];
  __shared__ double red[kQThreads / 32];
  const int64_t row = blockIdx.x;
  const char* base = static_cast<const char*>(in) + row * in_stride * 4;
  // the reference z-scores float32 data (integer rows converted exactly)
  auto xv = [&](int64_t i) -> float {
    return kind == SPP_OUT_I32 ? (float)reinterpret_cast<const int32_t*>(base)[i]
                               : reinterpret_cast<const float*>(base)[i];
  };
  const int64_t r0 = (n - 1) / 2, r1 = n / 2;
  select_pair<uint32_t>(n, r0, r1, [&](int64_t i) { return f32_key(xv(i)); }, hist, k32);
  const float a = key_f32(k32[0]), b = key_f32(k32[1]);
  const float med32 = (n & 1) ? a : __fmul_rn(__fadd_rn(a, b), 0.5f);
  const double med64 = (n & 1) ? (double)a : __dmul_rn(__dadd_rn((double)a, (double)b), 0.5);
  select_pair<unsigned long long>(
      n, r0, r1,
      [&](int64_t i) {
        return (unsigned long long)__double_as_longlong(fabs(__dsub_rn((double)xv(i), med64)));
      },
      hist, k64);
  const double da = __longlong_as_double((long long)k64[0]);
  const double db = __longlong_as_double((long long)k64[1]);
  const double medd = (n & 1) ? da : __dmul_rn(__dadd_rn(da, db), 0.5);
  double mad = __ddiv_rn(medd, 0.6744897501960817);  // scipy.stats.norm.ppf(0.75)
  if (fabs(mad) <= 1e-8) {  // np.isclose(mad, 0)
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += fabs(__dsub_rn((double)xv(i), med64));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kQThreads / 32; ++w) t += red[w];
      mad = __ddiv_rn(__ddiv_rn(t, (double)n), __dsqrt_rn(__ddiv_rn(2.0, 3.141592653589793)));
    }
  }
  if (threadIdx.x == 0) {
    locscale[row * 2] = (double)med32;
    locscale[row * 2 + 1] = fabs(mad) <= 1e-8 ? 1.0 : mad;
  }
}

extern "C" {

int spp_boxcar_snr(const void* in, int in_kind, int64_t nrows, int64_t n, int64_t in_stride,
                   const int32_t* factors, int nfactors, const int32_t* widths, int nwidths,
                   float* snr, int32_t* peak_index, void* workspace, int64_t workspace_bytes,
                   void* stream) {
  return boxcar_snr_impl(in, in_kind, nrows, n, in_stride, factors, nfactors, widths, nwidths, snr,
                         peak_index, workspace, workspace_bytes, stream, false);
}

int spp_boxcar_filter(const float* in, int64_t n, int width, float* out, void* stream) {
  if (!in || !out) return fail(SPP_ERR_ARG, "spp_boxcar_filter: null pointer");
  if (width < 1) return fail(SPP_ERR_ARG, "invalid boxcar width: %d", width);
  if (n <= 0) return fail(SPP_ERR_ARG, "empty series");
  if (width > 8192) return fail(SPP_ERR_UNSUPPORTED, "boxcar width %d > 8192", width);
  if (in == out) return fail(SPP_ERR_ARG, "spp_boxcar_filter: in and out must differ");
  const int64_t pad_left = width / 2;
  // the reference's -width // 2 + 1 (odd) or -width // 2 (even), Python floor
  // division: -(width / 2) either way
  const int64_t ref_bin = -(int64_t)(width / 2);
  const int64_t smem = (int64_t)(kBoxT + width - 1) * 4;
  int rc = SPP_OK;
  if (smem > 48 * 1024) {
    rc = set_smem_attr(reinterpret_cast<const void*>(k_boxcar_filter), smem);
    if (rc) return rc;
  }
  k_boxcar_filter<<<(unsigned)ceil_div(n, kBoxT), kBoxThreads, smem, as_stream(stream)>>>(
      in, n, width, pad_left, ref_bin, out);
  return cuda_status(cudaGetLastError(), "boxcar filter launch");
}

int spp_row_loc_scale(const void* in, int in_kind, int64_t nrows, int64_t n, int64_t in_stride,
                      int method, double* loc_scale, void* stream) {
  if (!in || !loc_scale) return fail(SPP_ERR_ARG, "spp_row_loc_scale: null pointer");
  if (in_kind != SPP_OUT_F32 && in_kind != SPP_OUT_I32) return fail(SPP_ERR_ARG, "bad in_kind");
  if (nrows <= 0 || nrows > 65535 || n <= 0) return fail(SPP_ERR_ARG, "bad sizes");
  cudaStream_t st = as_stream(stream);
  if (method == 0) {
    k_row_mean_std<<<(unsigned)nrows, 256, 0, st>>>(in, in_kind, n, in_stride, loc_scale);
    return cuda_status(cudaGetLastError(), "mean/std launch");
  }
  if (method == 2) {
    k_row_mad<<<(unsigned)nrows, kQThreads, 0, st>>>(in, in_kind, n, in_stride, loc_scale);
    return cuda_status(cudaGetLastError(), "median/MAD launch");
  }
  if (method != 1)
    return fail(SPP_ERR_ARG, "method must be 0 (mean/std), 1 (median/iqr) or 2 (median/mad)");
  SnrCfg cfg{};
  cfg.nf = 1;
  cfg.f[0] = 1;
  const int64_t qsmem = (int64_t)kQRanks * kQBins * 4;
  int rc = set_smem_attr(reinterpret_cast<const void*>(k_row_quantiles), qsmem);
  if (rc) return rc;
  k_row_quantiles<<<(unsigned)nrows, kQThreads, qsmem, st>>>(in, in_kind, n, in_stride, cfg,
                                                             loc_scale);
  return cuda_status(cudaGetLastError(), "row quantiles launch");
}

int spp_zscore(const float* in, int64_t n, const double* loc_scale, float* out, void* stream) {
  if (!in || !loc_scale || !out) return fail(SPP_ERR_ARG, "spp_zscore: null pointer");
  if (n <= 0) return fail(SPP_ERR_ARG, "empty series");
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 16);
  k_zscore<<<blocks, 256, 0, as_stream(stream)>>>(in, n, loc_scale, out);
  return cuda_status(cudaGetLastError(), "zscore launch");
}

int spp_matched_filter(const float* z, int64_t n, int64_t nfft, const double* temps,
                       const int32_t* temp_offsets, const int32_t* ref_bins,
                       const double* temp_stats, int ntemps, float* convs, void* workspace,
                       int64_t workspace_bytes, void* stream) {
  if (!z || !temps || !temp_offsets || !ref_bins || !temp_stats || !convs || !workspace)
    return fail(SPP_ERR_ARG, "spp_matched_filter: null pointer");
  if (n <= 0 || nfft < n) return fail(SPP_ERR_ARG, "need 0 < n <= nfft");
  if (ntemps <= 0 || ntemps > 65535) return fail(SPP_ERR_ARG, "bad template count");
  if (workspace_bytes < 16) return fail(SPP_ERR_SIZE, "workspace < 16 B");
  if ((int64_t)ntemps * n > 0xFFFFFFFFll) return fail(SPP_ERR_UNSUPPORTED, "ntemps * n >= 2^32");
  cudaStream_t st = as_stream(stream);
  double* spad = static_cast<double*>(workspace);
  unsigned long long* best = reinterpret_cast<unsigned long long*>(spad + 1);
  int rc = cuda_status(cudaMemsetAsync(best, 0, 8, st), "best clear");
  if (rc) return rc;
  k_padded_sum<<<1, 1024, 0, st>>>(z, n, nfft, spad);
  rc = cuda_status(cudaGetLastError(), "padded sum launch");
  if (rc) return rc;
  dim3 grid((unsigned)ceil_div(n, 256), (unsigned)ntemps);
  k_template_conv<<<grid, 256, 0, st>>>(z, n, nfft, temps, temp_offsets, ref_bins, temp_stats,
                                        spad, convs);
  rc = cuda_status(cudaGetLastError(), "template convolution launch");
  if (rc) return rc;
  const int64_t count = (int64_t)ntemps * n;
  k_argmax_first<<<(unsigned)std::min<int64_t>(ceil_div(count, 256), 148 * 8), 256, 0, st>>>(
      convs, count, best);
  return cuda_status(cudaGetLastError(), "argmax launch");
}

int64_t spp_boxcar_snr_robust_workspace_bytes(int64_t nrows, int64_t n, int nfactors,
                                              int nwidths) {
  int64_t nck;
  return snr_ws(nrows, n, nfactors, nwidths, &nck) + round_up(nrows * nfactors * 16, 256);
}

int spp_boxcar_snr_robust(const void* in, int in_kind, int64_t nrows, int64_t n,
                          int64_t in_stride, const int32_t* factors, int nfactors,
                          const int32_t* widths, int nwidths, float* snr, int32_t* peak_index,
                          void* workspace, int64_t workspace_bytes, void* stream) {
  return boxcar_snr_impl(in, in_kind, nrows, n, in_stride, factors, nfactors, widths, nwidths, snr,
                         peak_index, workspace, workspace_bytes, stream, true);
}

}  // extern "C"
