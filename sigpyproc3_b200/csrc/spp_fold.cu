// Folding (kernels.fold, core/kernels.py:403-445): every channel's delayed
// sample of one read_plan block is added into the (subintegration, subband,
// phase bin) cell its time falls in, and counted.
//
// One thread per (sample, subband): it derives the sample's phase bin and
// subintegration with the reference's float64 arithmetic -- same operations in
// the same order, each rounded (no fused multiply-adds), Python's float floor
// division -- sums the subband's channels and adds the sum and the channel
// count into the cell with one atomic each.  Float32 cells (spp_fold) are
// order-dependent in their last bits for float32 data, and for 8-bit data once
// a cell passes 2^24; the 8-bit form with 64-bit integer cells
// (spp_fold_exact) is exact and deterministic for any length.
#include <cmath>

#include "spp_common.cuh"

namespace spp {

// Python's float a // b (CPython's fmod-based floor division), restated.
__device__ __forceinline__ double py_floordiv(double a, double b) {
  const double mod = fmod(a, b);
  double div = __ddiv_rn(__dsub_rn(a, mod), b);
  if (mod != 0.0 && ((b < 0.0) != (mod < 0.0))) div = __dsub_rn(div, 1.0);
  if (div == 0.0) return copysign(0.0, __ddiv_rn(a, b));
  double fl = floor(div);
  if (__dsub_rn(div, fl) > 0.5) fl = __dadd_rn(fl, 1.0);
  return fl;
}

struct FoldArgs {
  const void* in;
  int is_f32;
  int64_t nchans, nsamps, nvalid;  // nvalid = samples of the block that are folded
  const int32_t* delays;
  const int32_t* band_start;  // nsubs + 1 channel boundaries
  double tsamp, period, accel, tobs, factor1;
  int64_t index;
  int32_t nbins, nsubs;
  float* fold_ar;
  unsigned long long* fold_u64;  // 8-bit exact cells (spp_fold_exact), else null
  int32_t* count_ar;
  int64_t cells;  // nints * nsubs * nbins
};

__global__ void k_fold(const FoldArgs a) {
  const int64_t isamp = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int band = blockIdx.y;
  if (isamp >= a.nvalid) return;
  // nbins * tj * (1 + accel * (tj - tobs) / (2 * c)) / period + 0.5, left to right
  const double tj = __dmul_rn((double)(isamp + a.index), a.tsamp);
  const double u = __ddiv_rn(__dmul_rn(a.accel, __dsub_rn(tj, a.tobs)), 2.0 * 299792458.0);
  const double t = __dmul_rn(__dmul_rn((double)a.nbins, tj), __dadd_rn(1.0, u));
  const double phase = __dadd_rn(__ddiv_rn(t, a.period), 0.5);
  const long long phasebin = llabs((long long)phase) % a.nbins;
  const double subint = py_floordiv((double)(isamp + a.index), a.factor1);
  const double pos1 =
      __dadd_rn(__dmul_rn(__dmul_rn(subint, (double)a.nbins), (double)a.nsubs), (double)phasebin);
  const int64_t pos2 = (int64_t)__dadd_rn(pos1, __dmul_rn((double)band, (double)a.nbins));
  if (pos2 < 0 || pos2 >= a.cells) return;  // unreachable for valid arguments; never write outside
  const int c0 = a.band_start[band], c1 = a.band_start[band + 1];
  if (c1 <= c0) return;
  // row of channel c: isamp + delay, a negative one wrapping to the block's end
  // (numba's negative index); rows outside the block are never read
  if (a.fold_u64) {  // 8-bit data, exact integer cells
    const uint8_t* x = static_cast<const uint8_t*>(a.in);
    unsigned long long s = 0;
    for (int c = c0; c < c1; ++c) {
      int64_t row = isamp + a.delays[c];
      if (row < 0) row += a.nsamps;
      if (row >= 0 && row < a.nsamps) s += x[a.nchans * row + c];
    }
    atomicAdd(a.fold_u64 + pos2, s);
    atomicAdd(a.count_ar + pos2, c1 - c0);
    return;
  }
  float sum;
  if (a.is_f32) {
    const float* x = static_cast<const float*>(a.in);
    float s = 0.f;
    for (int c = c0; c < c1; ++c) {
      int64_t row = isamp + a.delays[c];
      if (row < 0) row += a.nsamps;
      if (row >= 0 && row < a.nsamps) s = __fadd_rn(s, x[a.nchans * row + c]);
    }
    sum = s;
  } else {
    const uint8_t* x = static_cast<const uint8_t*>(a.in);
    int s = 0;
    for (int c = c0; c < c1; ++c) {
      int64_t row = isamp + a.delays[c];
      if (row < 0) row += a.nsamps;
      if (row >= 0 && row < a.nsamps) s += x[a.nchans * row + c];
    }
    sum = (float)s;
  }
  atomicAdd(a.fold_ar + pos2, sum);
  atomicAdd(a.count_ar + pos2, c1 - c0);
}

}  // namespace spp

using namespace spp;

static int fold_impl(const void* in, int nbits, int64_t nchans, int64_t nsamps,
                     const int32_t* delays, int32_t maxdelay, float tsamp, float period,
                     float accel, int64_t total_nsamps, int32_t nbins, int32_t nints,
                     int32_t nsubs, int64_t index, const int32_t* band_start, float* fold_ar,
                     unsigned long long* fold_u64, int32_t* count_ar, int64_t cells,
                     void* stream) {
  if (!in || !delays || !band_start || (!fold_ar && !fold_u64) || !count_ar)
    return fail(SPP_ERR_ARG, "spp_fold: null pointer");
  if (nbits != 8 && nbits != 32)
    return fail(SPP_ERR_UNSUPPORTED, "spp_fold takes 8-bit or float32 samples (unpack first)");
  if (nchans <= 0 || nbins <= 0 || nints <= 0 || nsubs <= 0 || nsubs > 65535 || maxdelay < 0)
    return fail(SPP_ERR_ARG, "spp_fold: bad shape");
  if (cells < (int64_t)nbins * nints * nsubs)
    return fail(SPP_ERR_SIZE, "spp_fold: %lld cells < nints * nsubs * nbins", (long long)cells);
  const int64_t nvalid = nsamps - maxdelay;
  if (nvalid <= 0) return SPP_OK;  // reference: range over a non-positive count
  if (index < 0 || index + nvalid > total_nsamps)
    return fail(SPP_ERR_ARG, "spp_fold: block [%lld, %lld) outside the %lld-sample observation",
                (long long)index, (long long)(index + nvalid), (long long)total_nsamps);
  FoldArgs a{};
  a.in = in;
  a.is_f32 = nbits == 32;
  a.nchans = nchans;
  a.nsamps = nsamps;
  a.nvalid = nvalid;
  a.delays = delays;
  a.band_start = band_start;
  // the reference receives tsamp, period and accel as float32
  a.tsamp = (double)tsamp;
  a.period = (double)period;
  a.accel = (double)accel;
  a.tobs = (double)total_nsamps * (double)tsamp;
  a.factor1 = (double)total_nsamps / (double)nints;
  a.index = index;
  a.nbins = nbins;
  a.nsubs = nsubs;
  a.fold_ar = fold_ar;
  a.fold_u64 = fold_u64;
  a.count_ar = count_ar;
  a.cells = cells;
  constexpr int kThreads = 256;
  const int64_t gx = ceil_div(nvalid, kThreads);
  if (gx > INT32_MAX) return fail(SPP_ERR_SIZE, "spp_fold: block too long");
  k_fold<<<dim3((unsigned)gx, (unsigned)nsubs), kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return cuda_status(cudaGetLastError(), "fold launch");
}

extern "C" int spp_fold(const void* in, int nbits, int64_t nchans, int64_t nsamps,
                        const int32_t* delays, int32_t maxdelay, float tsamp, float period,
                        float accel, int64_t total_nsamps, int32_t nbins, int32_t nints,
                        int32_t nsubs, int64_t index, const int32_t* band_start, float* fold_ar,
                        int32_t* count_ar, int64_t cells, void* stream) {
  return fold_impl(in, nbits, nchans, nsamps, delays, maxdelay, tsamp, period, accel,
                   total_nsamps, nbins, nints, nsubs, index, band_start, fold_ar, nullptr,
                   count_ar, cells, stream);
}

extern "C" int spp_fold_exact(const void* in, int64_t nchans, int64_t nsamps,
                              const int32_t* delays, int32_t maxdelay, float tsamp, float period,
                              float accel, int64_t total_nsamps, int32_t nbins, int32_t nints,
                              int32_t nsubs, int64_t index, const int32_t* band_start,
                              unsigned long long* fold_sums, int32_t* count_ar, int64_t cells,
                              void* stream) {
  return fold_impl(in, 8, nchans, nsamps, delays, maxdelay, tsamp, period, accel, total_nsamps,
                   nbins, nints, nsubs, index, band_start, nullptr, fold_sums, count_ar, cells,
                   stream);
}
