// Single-pass single-DM dedispersion for 8-bit data (the Filterbank.dedisperse
// hot loop, kernels.dedisperse core/kernels.py:340-362): raw time-major bytes
// go straight from HBM into shared memory, no corner turn.
//
// CTA = 256 output samples [t0, t0 + 256) over all channels, walked in slabs
// of 32 channels (32 bytes of each raw row).  All warps first read the delays
// of every slab in parallel (one round trip) into shared tables.  Slabs are
// then staged in packs: as many consecutive slabs as fit the row budget, each
// slab's rows [t0 + dmin_s, t0 + 256 + dmax_s) copied with 4-byte cp.async
// into shared rows of 36 bytes (pitch 9 words: the 32 consecutive rows a warp
// reads for one channel fall in 32 different banks); rows outside the block
// wrap once (numba's negative-index wraparound) or read as zero.  Each thread
// accumulates one output sample over all channels (exact int32) and stores it
// once.
#include <algorithm>

#include "spp_common.cuh"

namespace spp {

constexpr int kS1T = 256;        // outputs per CTA
constexpr int kS1Slab = 32;      // channels per slab
constexpr int kS1Pitch = 36;     // bytes per staged row

__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool valid) {
  const uint32_t d = smem_addr(dst);
  const int n = valid ? 4 : 0;  // src-size 0 fills zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

struct S1Args {
  const uint8_t* raw;
  int64_t nchans, nsamps;
  const int32_t* delays;
  int32_t dlo, dhi;
  float* out;
  int64_t out_start, nvalid;
  uint32_t* status;
};

// Per-slab delay range (every warp computes it from the same 32 delays).
__device__ __forceinline__ void slab_range(const S1Args& a, int c0, int lane, int32_t& d_lane,
                                           int32_t& mn, int32_t& mx) {
  const int c = c0 + lane;
  int32_t d = 0;
  if (c < a.nchans) {
    d = __ldg(a.delays + c);
    if (d < a.dlo || d > a.dhi) {
      dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)c);
      d = min(max(d, a.dlo), a.dhi);
    }
  }
  d_lane = d;
  mn = (c < a.nchans) ? d : INT32_MAX;
  mx = (c < a.nchans) ? d : INT32_MIN;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
}

// Stage rows [r0, r0 + nrows) of the slab starting at channel c0 into buf.
// Thread (row phase tid/8, word tid%8) walks rows 32 apart; rows inside the
// block use plain pointer increments, rows outside it wrap or read zero.
__device__ __forceinline__ void stage(const S1Args& a, uint8_t* buf, int64_t r0, int nrows, int c0) {
  const int64_t rowbytes = a.nchans;
  const int nw = min(kS1Slab, (int)(a.nchans - c0)) / 4;  // words per row (nchans % 4 == 0)
  const int w = threadIdx.x & 7;
  int r = threadIdx.x >> 3;
  constexpr int kStep = kS1T / 8;  // rows per pass
  if (w >= nw) return;
  if (r0 >= 0 && r0 + nrows <= a.nsamps) {
    const uint8_t* src = a.raw + (r0 + r) * rowbytes + c0 + 4 * w;
    uint8_t* dst = buf + r * kS1Pitch + 4 * w;
    const int64_t sstep = (int64_t)kStep * rowbytes;
    for (; r < nrows; r += kStep, src += sstep, dst += kStep * kS1Pitch) cp_async4(dst, src, true);
    return;
  }
  for (; r < nrows; r += kStep) {
    int64_t row = r0 + r;
    if (row < 0) row += a.nsamps;
    else if (row >= a.nsamps) row -= a.nsamps;
    const bool ok = row >= 0 && row < a.nsamps;
    const uint8_t* src = ok ? a.raw + row * rowbytes + c0 + 4 * w : a.raw;
    cp_async4(buf + r * kS1Pitch + 4 * w, src, ok);
  }
}

__global__ void __launch_bounds__(kS1T) k_dedisp_single8(const S1Args a, int32_t cap_rows) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int nslab = (int)((a.nchans + kS1Slab - 1) / kS1Slab);
  uint8_t* rowbuf = sm;
  int32_t* smn = reinterpret_cast<int32_t*>(sm + (int64_t)cap_rows * kS1Pitch);  // [nslab]
  int32_t* snr = smn + nslab;                                                    // [nslab] rows
  int32_t* sdo = snr + nslab;                                                    // [nslab][32]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t0 = (int64_t)blockIdx.x * kS1T;
  for (int sl = warp; sl < nslab; sl += kS1T / 32) {
    int32_t dl, mn, mx;
    slab_range(a, sl * kS1Slab, lane, dl, mn, mx);
    sdo[sl * 32 + lane] = (dl - mn) * kS1Pitch + lane;  // byte offset of channel lane
    if (lane == 0) {
      smn[sl] = mn;
      snr[sl] = kS1T + (mx - mn);
    }
  }
  __syncthreads();
  const int t = threadIdx.x;
  int32_t acc = 0;
  int s0 = 0;
  while (s0 < nslab) {
    // pack consecutive slabs into the row budget
    int s1 = s0, used = 0;
    while (s1 < nslab && used + snr[s1] <= cap_rows) used += snr[s1++];
    if (s1 == s0) {  // one slab larger than the budget: flag and stop
      if (t == 0) dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)s0);
      return;
    }
    int off = 0;
    for (int sl = s0; sl < s1; ++sl) {
      stage(a, rowbuf + (int64_t)off * kS1Pitch, t0 + smn[sl], snr[sl], sl * kS1Slab);
      off += snr[sl];
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    off = 0;
    for (int sl = s0; sl < s1; ++sl) {
      const uint8_t* base = rowbuf + (int64_t)(off + t) * kS1Pitch;
      const int32_t* dd = sdo + sl * 32;
      const int64_t rem = a.nchans - (int64_t)sl * kS1Slab;
      int32_t sacc = 0;
      if (rem >= kS1Slab) {
#pragma unroll
        for (int c = 0; c < kS1Slab; ++c) sacc += base[dd[c]];
      } else {
        for (int c = 0; c < (int)rem; ++c) sacc += base[dd[c]];
      }
      acc += sacc;
      off += snr[sl];
    }
    __syncthreads();
    s0 = s1;
  }
  const int64_t tt = t0 + t;
  if (tt < a.nvalid) a.out[a.out_start + tt] = (float)acc;
}

// Launches the single-pass kernel when it applies (8-bit, nchans % 4 == 0,
// every slab's rows within the shared-memory budget); returns
// SPP_ERR_UNSUPPORTED to let the caller use the corner-turn path otherwise.
int launch_single8(const uint8_t* raw, int64_t nchans, int64_t nsamps, const int32_t* delays,
                   int32_t dlo, int32_t dhi, float* out, int64_t out_start, int64_t nvalid,
                   uint32_t* status, cudaStream_t st) {
  if (nchans % 4 != 0 || (reinterpret_cast<uintptr_t>(raw) & 3) != 0 || nchans > 8192)
    return SPP_ERR_UNSUPPORTED;
  const int64_t nslab = ceil_div(nchans, kS1Slab);
  // a slab never needs more than kS1T + (dhi - dlo) rows
  const int64_t cap = std::max<int64_t>(1600, kS1T + ((int64_t)dhi - dlo) + 1);
  const int64_t smem = cap * kS1Pitch + nslab * (2 + 32) * 4;
  if (smem > 110 * 1024) return SPP_ERR_UNSUPPORTED;
  int rc = set_smem_attr(reinterpret_cast<const void*>(k_dedisp_single8), smem);
  if (rc) return rc;
  S1Args a{raw, nchans, nsamps, delays, dlo, dhi, out, out_start, nvalid, status};
  const int64_t gx = ceil_div(nvalid, kS1T);
  if (gx > INT32_MAX) return SPP_ERR_UNSUPPORTED;
  k_dedisp_single8<<<(unsigned)gx, kS1T, smem, st>>>(a, (int32_t)cap);
  return cuda_status(cudaGetLastError(), "single-DM launch");
}

}  // namespace spp
