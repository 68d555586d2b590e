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

// ---------------------------------------------------------------------------
// Host-table variant (spp_dedisperse_hd): the delays are known on the host, so
// every per-slab row range and per-channel byte offset is computed there and
// passed in the kernel parameters.  A CTA issues the copies of all its slabs
// at once -- one cp.async group per slab, no delay round trip first -- and
// adds slab s as soon as group s has landed.
//
// Staged rows are the raw 32 bytes of a slab, dense (16-B cp.async.cg).  A warp
// covers 4 consecutive outputs x 8 channel words per load: lane (i = lane & 3,
// j = lane >> 2) reads channel 4j + k of output row t + i.  For any delays the
// 32 lanes hit 32 distinct banks (bank = 8 * (row mod 4) + j), so every load
// is one wavefront.  Each lane keeps G partial sums (outputs 4g + i of its
// warp's range, over its channels); three shuffles over j finish them.  A CTA
// of W warps covers T = 4 W G outputs; W is chosen per launch (up to 32) so
// that one CTA per SM covers the block.
// Used when nchans is a multiple of 32, at most 32 * NS, and all slabs of a CTA
// fit in shared memory together.

constexpr int kHdMaxWarps = 32;
constexpr int kHdMaxG = 8;                    // output groups of 4 per warp
constexpr int kHdPitch = 32;                  // bytes per staged row

template <int NS>
struct S2Args {
  const uint8_t* raw;
  int64_t nchans, nsamps;
  float* out;
  int64_t out_start, nvalid;
  int32_t nslab;
  int32_t tab_off;       // byte offset of the channel-offset table in shared memory
  int32_t mn[NS];        // per slab: min delay
  int32_t nrows[NS];     // per slab: T + max - min rows staged
  int32_t srow[NS];      // per slab: first staged row in shared memory
  int32_t off[NS * 32];  // per channel: (delay - slab min) * 32 + channel in slab
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  const uint32_t d = smem_addr(dst);
  const int n = valid ? 16 : 0;  // src-size 0 fills zeros
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n)
               : "memory");
}

// Stage rows [r0, r0 + nrows) of the 32-channel slab at c0 with cp.async: two
// 16-B chunks per row, chunk q = 2 * row + half, threads striding by the block
// size; rows outside the block wrap once (numba negative indices) or read 0.
__device__ __forceinline__ void stage_hd(const uint8_t* raw, int64_t rowbytes, int64_t nsamps,
                                         uint8_t* buf, int64_t r0, int nrows, int64_t c0) {
  const int nq = 2 * nrows;
  const int nt = blockDim.x;  // a multiple of 32: every thread keeps its half
  int q = threadIdx.x;
  const int h = q & 1;
  const int row_step = nt >> 1;
  if (r0 >= 0 && r0 + nrows <= nsamps) {
    const uint8_t* src = raw + (r0 + (q >> 1)) * rowbytes + c0 + 16 * h;
    uint8_t* dst = buf + (q >> 1) * kHdPitch + 16 * h;
    const int64_t sstep = (int64_t)row_step * rowbytes;
    for (; q < nq; q += nt, src += sstep, dst += row_step * kHdPitch) cp_async16(dst, src, true);
    return;
  }
  for (; q < nq; q += nt) {
    int64_t row = r0 + (q >> 1);
    if (row < 0) row += nsamps;
    else if (row >= nsamps) row -= nsamps;
    const bool ok = row >= 0 && row < nsamps;
    const uint8_t* src = ok ? raw + row * rowbytes + c0 + 16 * h : raw;
    cp_async16(buf + (q >> 1) * kHdPitch + 16 * h, src, ok);
  }
}

// cp.async.wait_group takes an immediate; with `n` known after unrolling the
// switch folds to the one instruction.
__device__ __forceinline__ void cp_async_wait_n(int n) {
  switch (n) {
#define SPP_WAIT_CASE(k) \
  case k:                \
    cp_async_wait<k>();  \
    break;
    SPP_WAIT_CASE(0) SPP_WAIT_CASE(1) SPP_WAIT_CASE(2) SPP_WAIT_CASE(3) SPP_WAIT_CASE(4)
    SPP_WAIT_CASE(5) SPP_WAIT_CASE(6) SPP_WAIT_CASE(7) SPP_WAIT_CASE(8) SPP_WAIT_CASE(9)
    SPP_WAIT_CASE(10) SPP_WAIT_CASE(11) SPP_WAIT_CASE(12) SPP_WAIT_CASE(13) SPP_WAIT_CASE(14)
    SPP_WAIT_CASE(15) SPP_WAIT_CASE(16) SPP_WAIT_CASE(17) SPP_WAIT_CASE(18) SPP_WAIT_CASE(19)
    SPP_WAIT_CASE(20) SPP_WAIT_CASE(21) SPP_WAIT_CASE(22) SPP_WAIT_CASE(23) SPP_WAIT_CASE(24)
    SPP_WAIT_CASE(25) SPP_WAIT_CASE(26) SPP_WAIT_CASE(27) SPP_WAIT_CASE(28) SPP_WAIT_CASE(29)
    SPP_WAIT_CASE(30) SPP_WAIT_CASE(31)
#undef SPP_WAIT_CASE
    default:
      cp_async_wait<0>();
  }
}

template <int NS, int G>
__global__ void __launch_bounds__(32 * kHdMaxWarps)
k_dedisp_single8_hd(const __grid_constant__ S2Args<NS> a) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int T = 4 * G * (int)(blockDim.x >> 5);
  const int64_t t0 = (int64_t)blockIdx.x * T;
  // channel offsets into shared memory (each lane reads the four of its word);
  // kernel parameters only, so this runs before the wait below
  int32_t* tab = reinterpret_cast<int32_t*>(sm + a.tab_off);
  for (int c = threadIdx.x; c < 32 * a.nslab; c += blockDim.x) tab[c] = a.off[c];
  // Programmatic dependent launch: the previous kernel in the stream may still
  // be finishing (this grid was allowed to launch early); wait until its
  // memory operations are complete and visible before reading the input or
  // writing the output.  Without the launch attribute this returns at once.
  asm volatile("griddepcontrol.wait;" ::: "memory");
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    if (s < a.nslab)
      stage_hd(a.raw, a.nchans, a.nsamps, sm + (int64_t)a.srow[s] * kHdPitch, t0 + a.mn[s],
               a.nrows[s], 32 * s);
    cp_async_commit();  // one group per slab (empty past nslab)
  }
  // the next kernel in the stream may start launching (it waits for this
  // grid's completion before touching memory)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = lane & 3, j = lane >> 2;
  const int obase = warp * 4 * G + i;  // this lane's first output row within the CTA
  int32_t acc[G];
#pragma unroll
  for (int g = 0; g < G; ++g) acc[g] = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    cp_async_wait_n(NS - 1 - s);  // groups of slabs > s may still be in flight
    __syncthreads();
    if (s < a.nslab) {
      const int4 o4 = *reinterpret_cast<const int4*>(tab + 32 * s + 4 * j);
      const uint8_t* base = sm + (int64_t)(a.srow[s] + obase) * kHdPitch;
      const uint8_t* p0 = base + o4.x;
      const uint8_t* p1 = base + o4.y;
      const uint8_t* p2 = base + o4.z;
      const uint8_t* p3 = base + o4.w;
      uint32_t v[4][G];  // all 4 G loads of the slab issued before any add
#pragma unroll
      for (int g = 0; g < G; ++g) {
        v[0][g] = p0[g * 4 * kHdPitch];
        v[1][g] = p1[g * 4 * kHdPitch];
        v[2][g] = p2[g * 4 * kHdPitch];
        v[3][g] = p3[g * 4 * kHdPitch];
      }
#pragma unroll
      for (int g = 0; g < G; ++g) acc[g] += (int32_t)(v[0][g] + v[1][g] + v[2][g] + v[3][g]);
    }
  }
  // sum over the 8 channel words (lanes with equal i), then lane (i, j) writes group g = j
#pragma unroll
  for (int g = 0; g < G; ++g) {
    acc[g] += __shfl_xor_sync(0xffffffffu, acc[g], 4);
    acc[g] += __shfl_xor_sync(0xffffffffu, acc[g], 8);
    acc[g] += __shfl_xor_sync(0xffffffffu, acc[g], 16);
  }
  int32_t mine = 0;
#pragma unroll
  for (int g = 0; g < G; ++g)
    if (g == j) mine = acc[g];
  const int64_t tt = t0 + obase + 4 * j;
  if (j < G && tt < a.nvalid) a.out[a.out_start + tt] = (float)mine;
}

template <int NS>
static void (*hd_kernel(int G))(const S2Args<NS>) {
  switch (G) {
    case 1: return k_dedisp_single8_hd<NS, 1>;
    case 2: return k_dedisp_single8_hd<NS, 2>;
    case 3: return k_dedisp_single8_hd<NS, 3>;
    case 4: return k_dedisp_single8_hd<NS, 4>;
    case 5: return k_dedisp_single8_hd<NS, 5>;
    case 6: return k_dedisp_single8_hd<NS, 6>;
    case 7: return k_dedisp_single8_hd<NS, 7>;
    default: return k_dedisp_single8_hd<NS, 8>;
  }
}

template <int NS>
static int launch_hd(const uint8_t* raw, int64_t nchans, int64_t nsamps, const int32_t* d,
                     float* out, int64_t out_start, int64_t nvalid, cudaStream_t st) {
  S2Args<NS> a{};
  const int nslab = (int)(nchans / 32);
  int32_t mn[NS], mx[NS];
  for (int s = 0; s < nslab; ++s) {
    mn[s] = *std::min_element(d + 32 * s, d + 32 * s + 32);
    mx[s] = *std::max_element(d + 32 * s, d + 32 * s + 32);
  }
  // outputs per CTA T = 4 W G: one wave of CTAs covers the block, G up to 4
  // and as many warps W (up to 32) as that takes; shrink W until every slab's
  // rows are resident at once.  Blocks of more than 148 x 1024 outputs run two
  // CTAs per SM (half the shared memory each), so that one CTA's copies
  // overlap the other's adds (measured: 2^20 x 256 ch, 99 -> 90 us; at 65 536
  // samples one CTA per SM is faster).
  const int cps = nvalid > 148 * 1024 ? 2 : 1;
  const int64_t kMaxSmem = cps == 1 ? 227 * 1024 : 112 * 1024;
  const int64_t tab_bytes = 32 * 4 * (int64_t)nslab;
  const int64_t target = ceil_div(nvalid, 148 * cps);
  const int G = (int)std::min<int64_t>(kHdMaxG, std::max<int64_t>(1, ceil_div(target, 4 * kHdMaxWarps)));
  int W = (int)std::min<int64_t>(kHdMaxWarps, std::max<int64_t>(1, ceil_div(target, 4 * G)));
  int64_t rows = 0;
  for (; W >= 1; --W) {
    rows = 0;
    for (int s = 0; s < nslab; ++s) rows += 4 * W * G + (int64_t)(mx[s] - mn[s]);
    if (rows * kHdPitch + tab_bytes <= kMaxSmem) break;
  }
  if (W < 1) return SPP_ERR_UNSUPPORTED;
  const int T = 4 * W * G;
  int64_t r = 0;
  for (int s = 0; s < nslab; ++s) {
    a.mn[s] = mn[s];
    a.nrows[s] = T + (mx[s] - mn[s]);
    a.srow[s] = (int32_t)r;
    r += a.nrows[s];
    for (int c = 0; c < 32; ++c) a.off[32 * s + c] = (d[32 * s + c] - mn[s]) * kHdPitch + c;
  }
  a.raw = raw;
  a.nchans = nchans;
  a.nsamps = nsamps;
  a.out = out;
  a.out_start = out_start;
  a.nvalid = nvalid;
  a.nslab = nslab;
  a.tab_off = (int32_t)(rows * kHdPitch);
  const int64_t smem = rows * kHdPitch + tab_bytes;
  auto fn = hd_kernel<NS>(G);
  int rc = set_smem_attr(reinterpret_cast<const void*>(fn), smem);
  if (rc) return rc;
  const int64_t gx = ceil_div(nvalid, T);
  if (gx > INT32_MAX || nsamps > INT32_MAX) return SPP_ERR_UNSUPPORTED;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)gx);
  cfg.blockDim = dim3(32 * W);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cuda_status(cudaLaunchKernelEx(&cfg, fn, a), "single-DM (host table) launch");
}

// 8-bit, nchans a multiple of 32 up to 1024, delays in host memory; returns
// SPP_ERR_UNSUPPORTED when the shape is outside what the kernel covers.
int launch_single8_hd(const uint8_t* raw, int64_t nchans, int64_t nsamps, const int32_t* delays_host,
                      float* out, int64_t out_start, int64_t nvalid, cudaStream_t st) {
  if (nchans % 32 != 0 || nchans <= 0 || (reinterpret_cast<uintptr_t>(raw) & 15) != 0)
    return SPP_ERR_UNSUPPORTED;
  if (nchans <= 256)
    return launch_hd<8>(raw, nchans, nsamps, delays_host, out, out_start, nvalid, st);
  if (nchans <= 512)
    return launch_hd<16>(raw, nchans, nsamps, delays_host, out, out_start, nvalid, st);
  if (nchans <= 1024)
    return launch_hd<32>(raw, nchans, nsamps, delays_host, out, out_start, nvalid, st);
  return SPP_ERR_UNSUPPORTED;
}

}  // namespace spp
