// Brute-force DM-time transform kernels (device code, templates).
//
// Data path
//   raw filterbank (time-major, nbits packed) --k_corner_turn--> "planar" rows
//   (channel-major, time along 32-bit words, nbits per sample, LSB-first)
//   --k_dmt--> out[dm][t] = sum_c planar[c][t + off(dm, c)]
//
// k_dmt: one CTA owns DW DM trials x T output samples.  It walks the channels
// in slabs of SLAB channels.  A producer warp stages, per channel, the
// 16-B-aligned window of that channel's planar row that the CTA's DMs touch
// (cp.async.bulk, completion on an mbarrier, STAGES-deep ring); DW*TW
// consumer warps each own one DM and 32*R words of time (R*spw samples per
// thread) and accumulate with SIMD-within-a-register adds (integer input) or
// compensated fp32 / fp64 (float input).  All waits are bounded.
#pragma once

#include "spp_common.cuh"

namespace spp {

// ----------------------------------------------------------------------------
// Planar layout: row c holds samples s in [-halo, nsamps + pad) at word
// (s + halo) / spw, bit ((s + halo) % spw) * NB.  halo is a multiple of 4*spw
// samples so rows start 16-B aligned; pitch_w is a multiple of 4 words.
// Samples outside [0, nsamps) wrap modulo nsamps (once), which reproduces
// numba's negative-index wraparound used by kernels.dedisperse and the
// circular roll of kernels.roll_block.
// ----------------------------------------------------------------------------
template <int NB>
struct Pack {
  static constexpr int kSpw = (NB == 32) ? 1 : 32 / NB;         // samples per word
  static constexpr int kLogSpw =
      (NB == 32) ? 0 : (NB == 1 ? 5 : NB == 2 ? 4 : NB == 4 ? 3 : NB == 8 ? 2 : 1);
  static constexpr uint32_t kMaskByte = (NB == 1)   ? 0x01010101u
                                        : (NB == 2) ? 0x03030303u
                                        : (NB == 4) ? 0x0F0F0F0Fu
                                                    : 0xFFFFFFFFu;
  static constexpr int kG = (NB >= 8) ? 1 : 8 / NB;  // samples per byte
  // channels that fit in a byte lane / a 16-bit lane before overflow
  static constexpr int kCap8 = (NB >= 8) ? 1 : 255 / ((1 << NB) - 1);
  static constexpr int kCap16 = (NB >= 16) ? 1 : 65535 / ((1 << NB) - 1);
};

// Extracts the NB-bit field of channel `c` from its packed byte (sigproc
// bit order: big = first channel in the most significant bits).
template <int NB>
__device__ __forceinline__ uint32_t field_of(uint32_t byte, int c, int bitorder) {
  if (NB == 8) return byte;
  constexpr int per = 8 / NB;
  const int p = c % per;
  const int sh = (bitorder == SPP_BITORDER_BIG) ? (8 - (p + 1) * NB) : (p * NB);
  return (byte >> sh) & ((1u << NB) - 1u);
}

// Maps a planar sample index to a raw row index (wrap once) or -1 (zero).
__device__ __forceinline__ int64_t wrap_row(int64_t s, int64_t nsamps) {
  if (s < 0) s += nsamps;
  else if (s >= nsamps) s -= nsamps;
  return (s >= 0 && s < nsamps) ? s : -1;
}

// ----------------------------------------------------------------------------
// Corner turn for packed integer data.  CTA = 64 channels x 16 planar words.
// Loads the raw rows (16*spw of them, wrapped) of its channel group into
// shared memory, builds one planar word per (channel, word) and writes rows
// of 16 words.
// ----------------------------------------------------------------------------
constexpr int kCtChans = 64;
constexpr int kCtWords = 16;
// Tile of the bit-plane corner turn: 256 / nb channels (32 bytes of each raw
// row: whole 32-byte sectors in) by kPlaneWords words of each plane row
// (8 words = 32 bytes: whole sectors out), i.e. 256 raw rows.
__host__ __device__ constexpr int planes_ct_chans(int nb) { return 256 / nb; }
constexpr int kPlaneWords = 8;

template <int NB>
__global__ void __launch_bounds__(256)
k_corner_turn_int(const uint8_t* __restrict__ raw, int64_t nchans, int64_t nsamps,
                  int bitorder, int64_t halo, uint32_t* __restrict__ planar,
                  int64_t pitch_w) {
  using P = Pack<NB>;
  constexpr int RT = kCtWords * P::kSpw;      // raw rows in the tile
  constexpr int SB = kCtChans * NB / 8;       // bytes per raw row segment (full tile)
  constexpr int SBP = SB + 4;                 // smem pitch
  __shared__ __align__(16) uint8_t s_raw[RT * SBP];
  __shared__ uint32_t s_out[kCtChans][kCtWords + 1];

  const int64_t c0 = (int64_t)blockIdx.x * kCtChans;
  const int nc = (int)((nchans - c0) < kCtChans ? (nchans - c0) : kCtChans);
  const int seg = (nc * NB + 7) / 8;
  const int64_t rowbytes = nchans * NB / 8;
  const int64_t segstart = c0 * NB / 8;
  const bool vec = ((rowbytes & 3) == 0) && ((segstart & 3) == 0) && ((seg & 3) == 0) &&
                   ((reinterpret_cast<uintptr_t>(raw) & 3) == 0);
  const int64_t ntw = (pitch_w + kCtWords - 1) / kCtWords;

  for (int64_t by = blockIdx.y; by < ntw; by += gridDim.y) {
    const int64_t w0 = by * kCtWords;
    // load the raw rows of this tile (wrapped once around the block)
    if (vec) {
      const int nw = seg >> 2;
      for (int idx = threadIdx.x; idx < RT * nw; idx += blockDim.x) {
        const int r = idx / nw, k = idx - r * nw;
        const int64_t row = wrap_row(w0 * P::kSpw + r - halo, nsamps);
        uint32_t v = 0;
        if (row >= 0) v = __ldg(reinterpret_cast<const uint32_t*>(raw + row * rowbytes + segstart) + k);
        *reinterpret_cast<uint32_t*>(s_raw + r * SBP + 4 * k) = v;
      }
    } else {
      for (int idx = threadIdx.x; idx < RT * seg; idx += blockDim.x) {
        const int r = idx / seg, k = idx - r * seg;
        const int64_t row = wrap_row(w0 * P::kSpw + r - halo, nsamps);
        s_raw[r * SBP + k] = (row >= 0) ? __ldg(raw + row * rowbytes + segstart + k) : 0;
      }
    }
    __syncthreads();
    // build planar words: lanes over channels (conflict-free byte reads)
    for (int idx = threadIdx.x; idx < kCtChans * kCtWords; idx += blockDim.x) {
      const int c = idx % kCtChans, w = idx / kCtChans;
      uint32_t v = 0;
      if (c < nc) {
        const int byte = (c * NB) / 8;
#pragma unroll
        for (int j = 0; j < P::kSpw; ++j) {
          const uint32_t b = s_raw[(w * P::kSpw + j) * SBP + byte];
          v |= field_of<NB>(b, c, bitorder) << (j * NB);
        }
      }
      s_out[c][w] = v;
    }
    __syncthreads();
    // store rows (lanes over words)
    for (int idx = threadIdx.x; idx < kCtChans * kCtWords; idx += blockDim.x) {
      const int w = idx % kCtWords, c = idx / kCtWords;
      if (c < nc && w0 + w < pitch_w) planar[(c0 + c) * pitch_w + w0 + w] = s_out[c][w];
    }
    __syncthreads();
  }
}

// IEEE-754 binary32 -> binary64 for normal numbers by field arithmetic:
// (-1)^s 2^(e-127) (1 + m 2^-23) is the binary64 number with the same sign,
// biased exponent e - 127 + 1023 = e + 896 and significand m followed by 29
// zero bits.  The high word is sign | (e + 896) << 20 | m >> 3, i.e.
// ((|u| >> 3) + (896 << 20)) | sign, and the low word m << 29 = u << 29.
// Integer-pipe work, so it runs beside the conversion unit's F2F; zero,
// subnormals, infinities and NaN are not handled (the caller checks
// f32_is_normal over its data first).
__device__ __forceinline__ bool f32_is_normal(float x) {
  return ((__float_as_uint(x) & 0x7fffffffu) - 0x00800000u) < 0x7f000000u;  // 1 <= e <= 254
}
__device__ __forceinline__ double f64_of_normal_f32(float x) {
  const uint32_t u = __float_as_uint(x);
  const uint32_t hi = (((u & 0x7fffffffu) >> 3) + (896u << 20)) | (u & 0x80000000u);
  return __hiloint2double((int)hi, (int)(u << 29));
}

// Corner turn for float32 data, optionally fused with zero-DM subtraction
// (kernels.remove_zerodm, core/kernels.py:465-505):
//   y = f32((f64(x) - zdm[t] * f64(chanwts[c])) + f64(bpass[c]))
// computed with round-to-nearest intrinsics (no contraction).  `special`
// (optional): set to 1 when any sample taken from the block (after zero-DM)
// is not a normal float32.
static __global__ void __launch_bounds__(256)
k_corner_turn_f32(const float* __restrict__ raw, int64_t nchans, int64_t nsamps,
                  int64_t halo, float* __restrict__ planar, int64_t pitch,
                  const double* __restrict__ zdm, const float* __restrict__ chanwts,
                  const float* __restrict__ bpass, uint32_t* __restrict__ special = nullptr) {
  __shared__ float tile[32][33];
  const int64_t c0 = (int64_t)blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const int64_t nty = (pitch + 31) / 32;
  bool odd = false;  // a sample from the block that is not a normal float32
  for (int64_t by = blockIdx.y; by < nty; by += gridDim.y) {
    const int64_t p0 = by * 32;  // planar column (sample + halo)
    for (int i = ty; i < 32; i += 8) {
      const int64_t row = wrap_row(p0 + i - halo, nsamps);
      const int64_t c = c0 + tx;
      float v = 0.f;
      if (row >= 0 && c < nchans) {
        v = __ldg(raw + row * nchans + c);
        if (zdm != nullptr) {
          const double t1 = __dmul_rn(zdm[row], (double)chanwts[c]);
          const double t2 = __dsub_rn((double)v, t1);
          v = (float)__dadd_rn(t2, (double)bpass[c]);
        }
        odd |= !f32_is_normal(v);
      }
      tile[i][tx] = v;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
      const int64_t c = c0 + i;
      const int64_t p = p0 + tx;
      if (c < nchans && p < pitch) planar[c * pitch + p] = tile[tx][i];
    }
    __syncthreads();
  }
  // every lane of every warp gets here (the loops above are uniform across a warp)
  if (special != nullptr && __any_sync(0xffffffffu, odd) && tx == 0) atomicOr(special, 1u);
}

// Per-sample zero-DM sums zdm[t] = sum_c f64(x[t][c]) (one warp per sample).
// zdm[t] = sum_c f64(x[t][c]), added in channel order (the order of the
// kernels.remove_zerodm loop, core/kernels.py:497-499): a warp owns 32 rows,
// stages 32 x 32 tiles through shared memory with coalesced loads, and each
// lane adds its row's channels one by one.
constexpr int kRowSumWarps = 8;
static __global__ void __launch_bounds__(kRowSumWarps * 32)
k_row_sum_f64(const float* __restrict__ raw, int64_t nchans, int64_t nsamps,
              double* __restrict__ zdm) {
  __shared__ float tile[kRowSumWarps][32][33];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t t0 = ((int64_t)blockIdx.x * kRowSumWarps + warp) * 32;
  if (t0 >= nsamps) return;
  double s = 0.0;
  for (int64_t c0 = 0; c0 < nchans; c0 += 32) {
    const int64_t c = c0 + lane;
    for (int r = 0; r < 32; ++r) {
      const int64_t t = t0 + r;
      tile[warp][r][lane] = (t < nsamps && c < nchans) ? __ldg(raw + t * nchans + c) : 0.f;
    }
    __syncwarp();
    const int nc = (nchans - c0) < 32 ? (int)(nchans - c0) : 32;
    for (int j = 0; j < nc; ++j) s = __dadd_rn(s, (double)tile[warp][lane][j]);
    __syncwarp();
  }
  if (t0 + lane < nsamps) zdm[t0 + lane] = s;
}

// ----------------------------------------------------------------------------
// Accumulators
// ----------------------------------------------------------------------------
// Integer NB in {1,2,4,8}: byte lanes (A) -> 16-bit lanes (E: bytes 0/2, O:
// bytes 1/3) -> 32-bit per-sample sums (S).  Byte lane i of A[k][g] holds the
// running sum of sample i*G + g of word k.
template <int NB, int R>
struct IntAcc {
  using P = Pack<NB>;
  static constexpr int G = P::kG;
  static constexpr int SPW = P::kSpw;
  uint32_t A[R][G];
  uint32_t E[R][G];
  uint32_t O[R][G];
  uint32_t S[R][SPW];

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < R; ++k) {
#pragma unroll
      for (int g = 0; g < G; ++g) A[k][g] = E[k][g] = O[k][g] = 0u;
#pragma unroll
      for (int j = 0; j < SPW; ++j) S[k][j] = 0u;
    }
  }
  __device__ __forceinline__ void add(uint32_t v, int k) {
    if (NB == 16) {
      S[k][0] += v & 0xFFFFu;
      S[k][1] += v >> 16;
    } else if (NB == 8) {
      E[k][0] += v & 0x00FF00FFu;
      O[k][0] += __byte_perm(v, 0u, 0x4341);  // bytes 1 and 3 into 16-bit lanes
    } else {
#pragma unroll
      for (int g = 0; g < G; ++g) A[k][g] += (v >> (g * NB)) & P::kMaskByte;
    }
  }
  __device__ __forceinline__ void flush8() {
    if (NB >= 8) return;
#pragma unroll
    for (int k = 0; k < R; ++k)
#pragma unroll
      for (int g = 0; g < G; ++g) {
        E[k][g] += A[k][g] & 0x00FF00FFu;
        O[k][g] += (A[k][g] >> 8) & 0x00FF00FFu;
        A[k][g] = 0u;
      }
  }
  __device__ __forceinline__ void flush16() {
    if (NB == 16) return;
#pragma unroll
    for (int k = 0; k < R; ++k)
#pragma unroll
      for (int g = 0; g < G; ++g) {
        S[k][0 * G + g] += E[k][g] & 0xFFFFu;
        S[k][2 * G + g] += E[k][g] >> 16;
        S[k][1 * G + g] += O[k][g] & 0xFFFFu;
        S[k][3 * G + g] += O[k][g] >> 16;
        E[k][g] = O[k][g] = 0u;
      }
  }
};

// ----------------------------------------------------------------------------
// DM-time transform kernel
// ----------------------------------------------------------------------------
struct DmtArgs {
  const void* planar;     // planar rows (uint32 words or floats)
  int64_t pitch_w;        // row pitch in words
  int64_t halo;           // samples of left halo
  int32_t nchans;
  const int32_t* delays;  // ndm x dpitch
  int64_t dpitch;
  int32_t ndm;
  int32_t sign;           // +1 dedisperse, -1 roll
  int32_t dlo, dhi;       // declared range of sign*delay
  int32_t span_max;       // max (dmax - dmin) over a DM tile and channel
  int32_t slot_w;         // words per channel per stage
  void* out;
  int32_t out_kind;
  int64_t out_stride;
  int64_t out_start;
  int64_t nvalid;
  uint32_t* status;
  // float64 accumulation of float32 rows: a word that is 0 when every sample
  // of the block is a normal float32 (set by the corner turn); then part of
  // the conversions run on the integer pipe.  nullptr: conversion unit only.
  const uint32_t* special;
  // channel-pair kernels (2-bit data): `planar` holds pair-sum rows of three
  // bit planes; per (DM tile, slab of pairs) the plan precomputes each DM's
  // decoded offsets (pair_off, DW x SLAB) and the rows to stage (pair_ent,
  // 2 x SLAB entries of (row, window start word relative to the tile; row -1:
  // unused))
  const int2* pair_off;
  const int2* pair_ent;
  int32_t npairs;
};

template <int NB, int R, int DW, int TW, int SLAB, int STAGES>
struct DmtShape {
  static constexpr int kSpw = Pack<NB>::kSpw;
  static constexpr int kNwc = DW * TW;                 // consumer warps
  static constexpr int kThreads = (kNwc + 1) * 32;     // + producer warp
  static constexpr int kT = TW * 32 * R * kSpw;        // samples per CTA tile
};

__host__ __device__ constexpr int64_t dmt_stage_bytes(int slab, int slot_w, int dw) {
  return (int64_t)slab * slot_w * 4 + (int64_t)dw * slab * 4 + (int64_t)slab * 4;
}

template <int NB, int R, int DW, int TW, int SLAB, int STAGES, int ACC>
__global__ void __launch_bounds__(DmtShape<NB, R, DW, TW, SLAB, STAGES>::kThreads)
k_dmt(const DmtArgs a) {
  using Sh = DmtShape<NB, R, DW, TW, SLAB, STAGES>;
  using P = Pack<NB>;
  constexpr int SPW = P::kSpw;
  constexpr int NWC = Sh::kNwc;
  constexpr int T = Sh::kT;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* sdata = reinterpret_cast<uint32_t*>(smem);
  int32_t* sdel = reinterpret_cast<int32_t*>(sdata + (int64_t)STAGES * SLAB * a.slot_w);
  int32_t* sbase = sdel + STAGES * DW * SLAB;  // reserved: window starts are folded into sdel
  uint64_t* full = reinterpret_cast<uint64_t*>(sbase + STAGES * SLAB + ((STAGES * SLAB) & 1));
  uint64_t* empty = full + STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int dm0 = blockIdx.x * DW;
  const int64_t t0 = (int64_t)blockIdx.y * T;
  const int nslab = (a.nchans + SLAB - 1) / SLAB;

  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NWC);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NWC) {
    // ---------------- producer warp ----------------
    const uint32_t* planar = static_cast<const uint32_t*>(a.planar);
    for (int k = 0; k < nslab; ++k) {
      const int s = k % STAGES;
      if (k >= STAGES && !mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, a.status)) break;
      const int c0 = k * SLAB;
      const int nc = min(SLAB, a.nchans - c0);
      int64_t ws_reg[(SLAB + 31) / 32];
#pragma unroll
      for (int jj = 0; jj < (SLAB + 31) / 32; ++jj) {
        const int j = lane + jj * 32;
        ws_reg[jj] = 0;
        if (j < nc) {
          const int c = c0 + j;
          int32_t dv[DW];
          int32_t mn = INT32_MAX, mx = INT32_MIN;
#pragma unroll
          for (int i = 0; i < DW; ++i) {
            const int dm = min(dm0 + i, a.ndm - 1);
            int32_t d = a.sign * __ldg(a.delays + (int64_t)dm * a.dpitch + c);
            if (d < a.dlo || d > a.dhi) {
              dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)c);
              d = min(max(d, a.dlo), a.dhi);
            }
            dv[i] = d;
            mn = min(mn, d);
            mx = max(mx, d);
          }
          if (mx - mn > a.span_max) {
            dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)c | 0x80000000u);
            mx = mn + a.span_max;
          }
          // each trial's sample offset from the start of the staged window
          const int64_t ws = ((t0 + mn + a.halo) / SPW) & ~int64_t(3);
          const int32_t base = (int32_t)(ws * SPW - a.halo - t0);
#pragma unroll
          for (int i = 0; i < DW; ++i) sdel[(s * DW + i) * SLAB + j] = min(dv[i], mx) - base;
          ws_reg[jj] = ws;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive_expect_tx(&full[s], (uint32_t)nc * a.slot_w * 4u);
      __syncwarp();
#pragma unroll
      for (int jj = 0; jj < (SLAB + 31) / 32; ++jj) {
        const int j = lane + jj * 32;
        if (j < nc)
          bulk_g2s(sdata + ((int64_t)s * SLAB + j) * a.slot_w,
                   planar + (int64_t)(c0 + j) * a.pitch_w + ws_reg[jj], a.slot_w * 4u, &full[s]);
      }
    }
    return;
  }

  // ---------------- consumer warps ----------------
  // Thread (warp (dmw, tw), lane) owns words wbase + lane + 32*r, r < R, of the
  // tile (interleaved across the warp so every shared-memory load of a warp
  // touches 32 consecutive words: no bank conflicts).
  const int dmw = warp / TW, tw = warp % TW;
  const int dm = dm0 + dmw;
  const int wbase = tw * 32 * R + lane;
  bool ok = true;

  if constexpr (NB == 32) {
    // float32 input
    float s_acc[R], c_acc[R];
    double d_acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) { s_acc[r] = 0.f; c_acc[r] = 0.f; d_acc[r] = 0.0; }
    // all samples normal: one word in four converts by field arithmetic
    // (integer pipe), the rest by F2F (conversion unit): exactly the same
    // values.  F2F alone keeps the conversion unit near full; the field
    // conversion costs ~6 issue slots, so half and half made the kernel
    // issue-bound at the same speed and one in four is the balance measured.
    const bool split = ACC == SPP_ACC_F64 && a.special != nullptr && *a.special == 0u;
    for (int k = 0; k < nslab; ++k) {
      const int s = k % STAGES;
      if (!mbar_wait(&full[s], (k / STAGES) & 1, a.status)) { ok = false; break; }
      const int nc = min(SLAB, a.nchans - k * SLAB);
      const float* sd = reinterpret_cast<const float*>(sdata) + (int64_t)s * SLAB * a.slot_w;
      const int32_t* dl = sdel + (s * DW + dmw) * SLAB;
      // SPP_ACC_KAHAN32: a plain fp32 partial over the slab (<= 32 channels),
      // then one compensated (Kahan) step per slab into the running sum
      float p_acc[R];
#pragma unroll
      for (int r = 0; r < R; ++r) p_acc[r] = 0.f;
      if (ACC == SPP_ACC_F64 && split) {
#pragma unroll 4
        for (int j = 0; j < nc; ++j) {
          const float* row = sd + j * a.slot_w + (wbase + dl[j]);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const float x = row[32 * r];
            d_acc[r] += (r % 4 == 3) ? f64_of_normal_f32(x) : (double)x;
          }
        }
      } else {
#pragma unroll 4
        for (int j = 0; j < nc; ++j) {
          const float* row = sd + j * a.slot_w + (wbase + dl[j]);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const float x = row[32 * r];
            if (ACC == SPP_ACC_F64) d_acc[r] += (double)x;
            else p_acc[r] = __fadd_rn(p_acc[r], x);
          }
        }
      }
      if (ACC != SPP_ACC_F64) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float y = __fsub_rn(p_acc[r], c_acc[r]);
          const float t = __fadd_rn(s_acc[r], y);
          c_acc[r] = __fsub_rn(__fsub_rn(t, s_acc[r]), y);
          s_acc[r] = t;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (!ok || dm >= a.ndm) return;
    float* out = static_cast<float*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t t = t0 + wbase + 32 * r;
      if (t < a.nvalid)
        out[t] = (ACC == SPP_ACC_F64) ? (float)d_acc[r] : __fsub_rn(s_acc[r], c_acc[r]);
    }
  } else {
    IntAcc<NB, R> acc;
    acc.zero();
    constexpr int K16 = (P::kCap16 / SLAB) > 0 ? (P::kCap16 / SLAB) : 1;
    constexpr int F8 = (P::kCap8 >= SLAB) ? SLAB : 16;  // byte-lane flush period (channels)
    static_assert(NB >= 8 || P::kCap8 >= F8, "byte lanes would overflow");
    static_assert(NB != 8 || P::kCap16 >= SLAB, "16-bit lanes would overflow");
    for (int k = 0; k < nslab; ++k) {
      const int s = k % STAGES;
      if (!mbar_wait(&full[s], (k / STAGES) & 1, a.status)) { ok = false; break; }
      const int nc = min(SLAB, a.nchans - k * SLAB);
      const uint32_t* sd = sdata + (int64_t)s * SLAB * a.slot_w;
      const int32_t* dl = sdel + (s * DW + dmw) * SLAB;
      for (int jb = 0; jb < nc; jb += F8) {
        const int je = min(nc, jb + F8);
#pragma unroll 4
        for (int j = jb; j < je; ++j) {
          const int o = dl[j];  // sample offset of the tile start in the slot
          const uint32_t* row = sd + j * a.slot_w + (o >> P::kLogSpw) + wbase;
          const int sh = (o & (SPW - 1)) * NB;
#pragma unroll
          for (int r = 0; r < R; ++r)
            acc.add(__funnelshift_r(row[32 * r], row[32 * r + 1], sh), r);
        }
        acc.flush8();
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (((k + 1) % K16) == 0) acc.flush16();
    }
    acc.flush16();
    if (!ok || dm >= a.ndm) return;
    if (a.out_kind == SPP_OUT_U16) {
      uint16_t* out = static_cast<uint16_t*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < SPW; ++j) {
          const int64_t t = t0 + (int64_t)(wbase + 32 * r) * SPW + j;
          if (t < a.nvalid) out[t] = (uint16_t)min(acc.S[r][j], 65535u);
        }
    } else if (a.out_kind == SPP_OUT_I32) {
      int32_t* out = static_cast<int32_t*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < SPW; ++j) {
          const int64_t t = t0 + (int64_t)(wbase + 32 * r) * SPW + j;
          if (t < a.nvalid) out[t] = (int32_t)acc.S[r][j];
        }
    } else {
      float* out = static_cast<float*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < SPW; ++j) {
          const int64_t t = t0 + (int64_t)(wbase + 32 * r) * SPW + j;
          if (t < a.nvalid) out[t] = (float)acc.S[r][j];
        }
    }
  }
}

// ----------------------------------------------------------------------------
// Persistent work-list DM-time kernel.  Each work item is one DM tile (up to
// DW rows) x one time tile of one (beam, channel group) with its own planar
// rows, delay rows and output rows, so uneven beams, chunk lengths and DM
// ranges run in a single launch.  CTAs stay resident (grid = a few per SM);
// the producer warp claims items from a global counter and streams their
// channel slabs through the STAGES-deep ring, tagging every stage with the
// item index; consumers follow the tags, so the ring never drains between
// items.  A tag of -1 ends the CTA.
// ----------------------------------------------------------------------------
struct DmtItem {
  const void* planar;     // first planar row of the channel group
  int64_t pitch_w;        // words per planar row
  int64_t halo;           // samples of left halo in the planar rows
  const int32_t* delays;  // delay row of the tile's first DM (rows dpitch apart)
  int64_t dpitch;
  void* out;              // output row of the tile's first DM
  int64_t out_stride;     // elements between output rows
  int64_t out_start;      // element offset of sample 0 in a row
  int64_t nvalid;         // samples to write per row
  int64_t t0;             // first output sample of the tile
  int32_t nchans;         // channels in the group
  int32_t nrows;          // DM rows in the tile (<= DW)
  int32_t sign;
  int32_t dlo, dhi;       // declared range of sign*delay
  int32_t span_max;
  int32_t out_kind;
  int32_t reserved;
};
static_assert(sizeof(DmtItem) == 112, "DmtItem layout is part of the C ABI");

struct WlArgs {
  const DmtItem* items;
  int32_t nitems;
  int32_t slot_w;
  int32_t* counter;  // zeroed before the launch
  uint32_t* status;
};

template <int NB, int R, int SPW>
__device__ __forceinline__ void store_int_outputs(const IntAcc<NB, R>& acc, const DmtItem& it,
                                                  int row, int64_t t0, int wbase) {
  if (it.out_kind == SPP_OUT_U16) {
    uint16_t* out = static_cast<uint16_t*>(it.out) + (int64_t)row * it.out_stride + it.out_start;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < SPW; ++j) {
        const int64_t t = t0 + (int64_t)(wbase + 32 * r) * SPW + j;
        if (t < it.nvalid) out[t] = (uint16_t)min(acc.S[r][j], 65535u);
      }
  } else if (it.out_kind == SPP_OUT_I32) {
    int32_t* out = static_cast<int32_t*>(it.out) + (int64_t)row * it.out_stride + it.out_start;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < SPW; ++j) {
        const int64_t t = t0 + (int64_t)(wbase + 32 * r) * SPW + j;
        if (t < it.nvalid) out[t] = (int32_t)acc.S[r][j];
      }
  } else {
    float* out = static_cast<float*>(it.out) + (int64_t)row * it.out_stride + it.out_start;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < SPW; ++j) {
        const int64_t t = t0 + (int64_t)(wbase + 32 * r) * SPW + j;
        if (t < it.nvalid) out[t] = (float)acc.S[r][j];
      }
  }
}

template <int NB, int R, int DW, int TW, int SLAB, int STAGES, int ACC>
__global__ void __launch_bounds__(DmtShape<NB, R, DW, TW, SLAB, STAGES>::kThreads)
k_dmt_wl(const WlArgs w) {
  using Sh = DmtShape<NB, R, DW, TW, SLAB, STAGES>;
  using P = Pack<NB>;
  constexpr int SPW = P::kSpw;
  constexpr int NWC = Sh::kNwc;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* sdata = reinterpret_cast<uint32_t*>(smem);
  int32_t* sdel = reinterpret_cast<int32_t*>(sdata + (int64_t)STAGES * SLAB * w.slot_w);
  int32_t* sbase = sdel + STAGES * DW * SLAB;  // reserved: window starts are folded into sdel
  int32_t* stag = sbase + STAGES * SLAB;  // per stage: item, slab, nslab, pad
  uint64_t* full = reinterpret_cast<uint64_t*>(stag + 4 * STAGES);
  uint64_t* empty = full + STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NWC);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NWC) {
    // ---------------- producer warp ----------------
    uint32_t gk = 0;
    bool ok = true;
    while (ok) {
      int it_idx = 0;
      if (lane == 0) it_idx = atomicAdd(w.counter, 1);
      it_idx = __shfl_sync(0xffffffffu, it_idx, 0);
      if (it_idx >= w.nitems) break;
      const DmtItem it = w.items[it_idx];
      const uint32_t* planar = static_cast<const uint32_t*>(it.planar);
      const int nslab = (it.nchans + SLAB - 1) / SLAB;
      for (int k = 0; k < nslab; ++k, ++gk) {
        const int s = gk % STAGES;
        if (gk >= STAGES && !mbar_wait(&empty[s], ((gk / STAGES) - 1) & 1, w.status)) {
          ok = false;
          break;
        }
        const int c0 = k * SLAB;
        const int nc = min(SLAB, it.nchans - c0);
        int64_t ws_reg[(SLAB + 31) / 32];
#pragma unroll
        for (int jj = 0; jj < (SLAB + 31) / 32; ++jj) {
          const int j = lane + jj * 32;
          ws_reg[jj] = 0;
          if (j < nc) {
            const int c = c0 + j;
            int32_t dv[DW];
            int32_t mn = INT32_MAX, mx = INT32_MIN;
#pragma unroll
            for (int i = 0; i < DW; ++i) {
              const int r = min(i, it.nrows - 1);
              int32_t d = it.sign * __ldg(it.delays + (int64_t)r * it.dpitch + c);
              if (d < it.dlo || d > it.dhi) {
                dev_flag(w.status, SPP_DEV_RANGE, (uint32_t)c);
                d = min(max(d, it.dlo), it.dhi);
              }
              dv[i] = d;
              mn = min(mn, d);
              mx = max(mx, d);
            }
            if (mx - mn > it.span_max) {
              dev_flag(w.status, SPP_DEV_RANGE, (uint32_t)c | 0x80000000u);
              mx = mn + it.span_max;
            }
            // each trial's sample offset from the start of the staged window
            const int64_t ws = ((it.t0 + mn + it.halo) / SPW) & ~int64_t(3);
            const int32_t base = (int32_t)(ws * SPW - it.halo - it.t0);
#pragma unroll
            for (int i = 0; i < DW; ++i) sdel[(s * DW + i) * SLAB + j] = min(dv[i], mx) - base;
            ws_reg[jj] = ws;
          }
        }
        if (lane == 0) {
          stag[4 * s + 0] = it_idx;
          stag[4 * s + 1] = k;
          stag[4 * s + 2] = nslab;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&full[s], (uint32_t)nc * w.slot_w * 4u);
        __syncwarp();
#pragma unroll
        for (int jj = 0; jj < (SLAB + 31) / 32; ++jj) {
          const int j = lane + jj * 32;
          if (j < nc)
            bulk_g2s(sdata + ((int64_t)s * SLAB + j) * w.slot_w,
                     planar + (int64_t)(c0 + j) * it.pitch_w + ws_reg[jj], w.slot_w * 4u, &full[s]);
        }
      }
    }
    if (ok) {
      const int s = gk % STAGES;
      if (gk < STAGES || mbar_wait(&empty[s], ((gk / STAGES) - 1) & 1, w.status)) {
        if (lane == 0) {
          stag[4 * s + 0] = -1;
          mbar_arrive(&full[s]);
        }
      }
    }
    return;
  }

  // ---------------- consumer warps ----------------
  // words wbase + lane + 32*r of the tile (interleaved: conflict-free loads)
  const int dmw = warp / TW, tw = warp % TW;
  const int wbase = tw * 32 * R + lane;
  uint32_t gk = 0;
  if constexpr (NB == 32) {
    float s_acc[R], c_acc[R];
    double d_acc[R];
    DmtItem it{};
    for (;; ++gk) {
      const int s = gk % STAGES;
      if (!mbar_wait(&full[s], (gk / STAGES) & 1, w.status)) return;
      const int it_idx = stag[4 * s + 0];
      if (it_idx < 0) return;
      const int k = stag[4 * s + 1], nslab = stag[4 * s + 2];
      if (k == 0) {
        it = w.items[it_idx];
#pragma unroll
        for (int r = 0; r < R; ++r) { s_acc[r] = 0.f; c_acc[r] = 0.f; d_acc[r] = 0.0; }
      }
      const int nc = min(SLAB, it.nchans - k * SLAB);
      const float* sd = reinterpret_cast<const float*>(sdata) + (int64_t)s * SLAB * w.slot_w;
      const int32_t* dl = sdel + (s * DW + dmw) * SLAB;
      // SPP_ACC_KAHAN32: a plain fp32 partial over the slab (<= 32 channels),
      // then one compensated (Kahan) step per slab into the running sum
      float p_acc[R];
#pragma unroll
      for (int r = 0; r < R; ++r) p_acc[r] = 0.f;
#pragma unroll 4
      for (int j = 0; j < nc; ++j) {
        const float* row = sd + j * w.slot_w + (wbase + dl[j]);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float x = row[32 * r];
          if (ACC == SPP_ACC_F64) d_acc[r] += (double)x;
          else p_acc[r] = __fadd_rn(p_acc[r], x);
        }
      }
      if (ACC != SPP_ACC_F64) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float y = __fsub_rn(p_acc[r], c_acc[r]);
          const float t = __fadd_rn(s_acc[r], y);
          c_acc[r] = __fsub_rn(__fsub_rn(t, s_acc[r]), y);
          s_acc[r] = t;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (k == nslab - 1 && dmw < it.nrows) {
        float* out = static_cast<float*>(it.out) + (int64_t)dmw * it.out_stride + it.out_start;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int64_t t = it.t0 + wbase + 32 * r;
          if (t < it.nvalid)
            out[t] = (ACC == SPP_ACC_F64) ? (float)d_acc[r] : __fsub_rn(s_acc[r], c_acc[r]);
        }
      }
    }
  } else {
    IntAcc<NB, R> acc;
    acc.zero();
    constexpr int K16 = (P::kCap16 / SLAB) > 0 ? (P::kCap16 / SLAB) : 1;
    constexpr int F8 = (P::kCap8 >= SLAB) ? SLAB : 16;
    DmtItem it{};
    for (;; ++gk) {
      const int s = gk % STAGES;
      if (!mbar_wait(&full[s], (gk / STAGES) & 1, w.status)) return;
      const int it_idx = stag[4 * s + 0];
      if (it_idx < 0) return;
      const int k = stag[4 * s + 1], nslab = stag[4 * s + 2];
      if (k == 0) {
        it = w.items[it_idx];
        acc.zero();
      }
      const int nc = min(SLAB, it.nchans - k * SLAB);
      const uint32_t* sd = sdata + (int64_t)s * SLAB * w.slot_w;
      const int32_t* dl = sdel + (s * DW + dmw) * SLAB;
      for (int jb = 0; jb < nc; jb += F8) {
        const int je = min(nc, jb + F8);
#pragma unroll 4
        for (int j = jb; j < je; ++j) {
          const int o = dl[j];
          const uint32_t* row = sd + j * w.slot_w + (o >> P::kLogSpw) + wbase;
          const int sh = (o & (SPW - 1)) * NB;
#pragma unroll
          for (int r = 0; r < R; ++r)
            acc.add(__funnelshift_r(row[32 * r], row[32 * r + 1], sh), r);
        }
        acc.flush8();
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (((k + 1) % K16) == 0) acc.flush16();
      if (k == nslab - 1) {
        acc.flush16();
        if (dmw < it.nrows) store_int_outputs<NB, R, SPW>(acc, it, dmw, it.t0, wbase);
      }
    }
  }
}

// ----------------------------------------------------------------------------
// Bit-sliced DM-time kernel for 1-, 2- and 4-bit data.
//
// Planar "plane rows": row c*NB + k holds bit k of channel c's samples, 32
// samples per word (LSB first).  A thread owns P words of time, interleaved
// across the warp (word = lane + 32*p, so a warp's loads hit 32 consecutive
// words: no bank conflicts).  Per channel it funnel-shifts each plane word to
// its delay and adds it, with weight 2^k, into a bit-sliced counter: word
// A[p][l] holds bit l of the 32 running sums.  Additions go through
// carry-save adders (three words in, sum and carry out; the carry-save
// popcount of Harley & Seal, as in Mula, Kurz & Lemire 2018), with at most
// one pending word per level, so a channel costs about four LOP3s per plane
// word.  The pending pattern over a full 64-channel slab is fixed, so the
// compiler resolves it statically.  L levels hold counts up to 2^L - 1.
// ----------------------------------------------------------------------------
// Carry-save adder: acc <- acc ^ x ^ y, carry <- majority(acc, x, y).
__device__ __forceinline__ void csa(uint32_t& acc, uint32_t x, uint32_t y, uint32_t& carry) {
  const uint32_t a = acc;
  acc = a ^ x ^ y;
  carry = (a & x) | (a & y) | (x & y);
}
// Half adder: acc <- acc ^ x, carry <- acc & x.
__device__ __forceinline__ void half(uint32_t& acc, uint32_t x, uint32_t& carry) {
  carry = acc & x;
  acc ^= x;
}

// Bit-sliced counter of 32 sums per word position p: A[p][l] holds bit l.
// Inputs arrive as four channels at a time (one word per plane and p); a
// fixed network of carry-save adders folds them in (levels 0..3 per four
// channels, 4..5 per sixteen, 6..7 per sixty-four) and the single carry that
// leaves each 64-channel slab ripples through the top levels with half adders.
template <int P, int L>
struct BitCounter {
  uint32_t A[P][L];

  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int l = 0; l < L; ++l) A[p][l] = 0u;
  }
  // Four channels of 2-bit samples: lo[q] weight 1, hi[q] weight 2.  Returns
  // (through out) the weight-16 carry word.
  __device__ __forceinline__ void quad2(int p, const uint32_t (&lo)[4], const uint32_t (&hi)[4],
                                        uint32_t& out16) {
    uint32_t ta, tb, fa, fb, fc, ea, eb;
    csa(A[p][0], lo[0], lo[1], ta);
    csa(A[p][0], lo[2], lo[3], tb);
    csa(A[p][1], hi[0], hi[1], fa);
    csa(A[p][1], hi[2], hi[3], fb);
    csa(A[p][1], ta, tb, fc);
    csa(A[p][2], fa, fb, ea);
    half(A[p][2], fc, eb);
    csa(A[p][3], ea, eb, out16);
  }
  // Four channels of 4-bit samples: x[b][q] is bit b (weight 2^b) of channel
  // q.  Per level: the four input words of that weight plus the carries from
  // the level below (2, 3, 4 and 4 of them).  Returns the weight-64 carry word.
  __device__ __forceinline__ void quad4(int p, const uint32_t (&x)[4][4], uint32_t& out64) {
    uint32_t c1a, c1b, c2a, c2b, c2c, c3a, c3b, c3c, c3d, c4a, c4b, c4c, c4d, c5a, c5b;
    csa(A[p][0], x[0][0], x[0][1], c1a);
    csa(A[p][0], x[0][2], x[0][3], c1b);
    csa(A[p][1], x[1][0], x[1][1], c2a);
    csa(A[p][1], x[1][2], x[1][3], c2b);
    csa(A[p][1], c1a, c1b, c2c);
    csa(A[p][2], x[2][0], x[2][1], c3a);
    csa(A[p][2], x[2][2], x[2][3], c3b);
    csa(A[p][2], c2a, c2b, c3c);
    half(A[p][2], c2c, c3d);
    csa(A[p][3], x[3][0], x[3][1], c4a);
    csa(A[p][3], x[3][2], x[3][3], c4b);
    csa(A[p][3], c3a, c3b, c4c);
    csa(A[p][3], c3c, c3d, c4d);
    csa(A[p][4], c4a, c4b, c5a);
    csa(A[p][4], c4c, c4d, c5b);
    csa(A[p][5], c5a, c5b, out64);
  }
  // Four channels of 1-bit samples.  Returns the weight-4 carry word.
  __device__ __forceinline__ void quad1(int p, const uint32_t (&x)[4], uint32_t& out4) {
    uint32_t ta, tb;
    csa(A[p][0], x[0], x[1], ta);
    csa(A[p][0], x[2], x[3], tb);
    csa(A[p][1], ta, tb, out4);
  }
  // Four words of weight 2^l -> accumulate at level l, l+1; carry of weight 2^(l+2).
  __device__ __forceinline__ void fold4(int p, int l, const uint32_t (&w)[4], uint32_t& out) {
    uint32_t a, b;
    csa(A[p][l], w[0], w[1], a);
    csa(A[p][l], w[2], w[3], b);
    csa(A[p][l + 1], a, b, out);
  }
  // Ripple a carry word of weight 2^l through the remaining levels.
  __device__ __forceinline__ void ripple(int p, int l, uint32_t c) {
#pragma unroll
    for (int k = 0; k < L; ++k) {
      if (k < l) continue;
      uint32_t nc;
      half(A[p][k], c, nc);
      c = nc;
    }
  }
  __device__ __forceinline__ uint32_t count(int p, int i) const {
    uint32_t v = 0;
#pragma unroll
    for (int l = 0; l < L; ++l) v |= ((A[p][l] >> i) & 1u) << l;
    return v;
  }
};

template <int NB, int P, int DW, int TW, int SLAB>
struct BitsShape {
  static constexpr int kNwc = DW * TW;
  static constexpr int kThreads = (kNwc + 1) * 32;
  static constexpr int kT = TW * 32 * P * 32;  // samples per CTA tile
};

// Shared memory per stage: SLAB channels x NB plane rows x slot_w words, plus
// DW x SLAB tile-relative sample offsets, each stored decoded as (word, bit
// shift) so the consumers spend no instructions splitting it.
__host__ __device__ constexpr int64_t bits_stage_bytes(int nb, int slab, int slot_w, int dw) {
  return (int64_t)slab * nb * slot_w * 4 + (int64_t)dw * slab * 8;
}

// Word layout of a thread's P words in the tile.  Odd P > 1: the P words are
// consecutive (lane stride P words, coprime with the 32 banks: conflict-free),
// so the P funnel shifts of a plane row need P + 1 shared loads; otherwise
// they are interleaved across the warp (lane + 32 p), 2 loads per word.
template <int P>
struct BitsWords {
  static constexpr bool kContig = (P & 1) && P > 1;
  __host__ __device__ static constexpr int base(int tw, int lane) {
    return kContig ? (tw * 32 + lane) * P : tw * 32 * P + lane;
  }
  __host__ __device__ static constexpr int pos(int p) { return kContig ? p : 32 * p; }
};

// Levels of the carry-save network per sample width: a quad of four channels
// leaves one carry word of weight 2^kQuad (4 x (2^NB - 1) < 2^kQuad); the
// counter needs kLevels levels for sums of 4096 channels (4096 x (2^NB - 1)
// < 2^kLevels for 1-, 2-, 4- and 8-bit samples).  NB = 3: sums of two 2-bit
// channels (0..6, three planes); 2048 of them need the 2-bit data's 14 levels.
template <int NB>
struct BitsLevels {
  static_assert(NB == 1 || NB == 2 || NB == 3 || NB == 4 || NB == 8,
                "bit-sliced kernels take 1-8 bit samples or 2-bit pair sums");
  static constexpr int kQuad = NB == 8 ? 10 : NB == 4 ? 6 : NB == 3 ? 5 : NB == 2 ? 4 : 2;
  static constexpr int kLevels = NB == 8 ? 20 : NB == 4 ? 16 : 14;
};

// Four channels of NB-bit samples through a carry-save network built level by
// level: level B takes the four plane-B words (fetched through word(b, q),
// aligned plane b of channel q, only when that level is reached, so few
// input words are live) and the carries from level B - 1, adds them into
// A[p][B] in pairs with carry-save adders (a half adder takes an odd one
// out) and passes one carry per adder up.  Above the top plane the carries
// are reduced the same way until one word is left: the carry of weight
// 2^kQuad.  For NB = 2 this is quad2's network, adder for adder.
template <int P, int L, int NB, int B, int NCIN>
struct QuadLevel {
  template <class F>
  __device__ __forceinline__ static void run(BitCounter<P, L>& c, int p, F& word,
                                             const uint32_t* cin, uint32_t& out) {
    constexpr int NP = B < NB ? 4 : 0;
    constexpr int NIN = NP + NCIN;
    constexpr int NOUT = (NIN + 1) / 2;
    uint32_t w[NIN];
#pragma unroll
    for (int q = 0; q < NP; ++q) w[q] = word(B, q);
#pragma unroll
    for (int k = 0; k < NCIN; ++k) w[NP + k] = cin[k];
    uint32_t co[NOUT];
#pragma unroll
    for (int k = 0; k < NIN / 2; ++k) csa(c.A[p][B], w[2 * k], w[2 * k + 1], co[k]);
    if constexpr (NIN & 1) half(c.A[p][B], w[NIN - 1], co[NOUT - 1]);
    if constexpr (NOUT == 1 && B + 1 >= NB) {
      static_assert(B + 1 == BitsLevels<NB>::kQuad, "quad carry level");
      out = co[0];
    } else {
      QuadLevel<P, L, NB, B + 1, NOUT>::run(c, p, word, co, out);
    }
  }
};

// One slab of SLAB channels through the carry-save network.  FULL: all
// channels present (no predicates); otherwise channels >= nc add zeros.
template <int NB, int P, int L, int SLAB, bool FULL, int SLOT = 0>
__device__ __forceinline__ void bits_slab(BitCounter<P, L>& cnt, const uint32_t* __restrict__ sd,
                                          const int2* __restrict__ off, int nc, int slot_rt,
                                          int wbase) {
  // SLOT > 0: slot width known at compile time (immediate load offsets)
  const int slot_w = SLOT > 0 ? SLOT : slot_rt;
  constexpr int NMID = SLAB / 16;
  uint32_t cmid[NMID][P];
#pragma unroll
  for (int m = 0; m < NMID; ++m) {  // 16 channels
    // the four quads' carries are folded pairwise as they arrive (quads 0+1
    // into pa, quads 2+3 then pa into the per-16-channel carry), so at most
    // two words per position are held
    uint32_t pa[P], pw[P];
#pragma unroll
    for (int i = 0; i < 4; ++i) {    // 4 channels
      // per channel: staged row start and bit shift, decoded once
      const uint32_t* base[4];
      int sh[4];
      bool live[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = 16 * m + 4 * i + q;
        live[q] = FULL || j < nc;
        const int2 ow = live[q] ? off[j] : make_int2(0, 0);  // (word, bit shift)
        sh[q] = ow.y;
        base[q] = sd + j * NB * slot_w + ow.x + wbase;
      }
      if constexpr (NB == 8) {
        // eight planes: each plane word is loaded when its level of the
        // network is reached (interleaved words: two loads per word)
        static_assert(!BitsWords<P>::kContig, "8-bit bit-sliced kernels use interleaved words");
#pragma unroll
        for (int p = 0; p < P; ++p) {
          auto word = [&](int b, int q) -> uint32_t {
            uint32_t lo = 0u, hi = 0u;
            if (live[q]) {
              lo = base[q][b * slot_w + 32 * p];
              hi = base[q][b * slot_w + 32 * p + 1];
            }
            return __funnelshift_r(lo, hi, sh[q]);
          };
          uint32_t cq;
          QuadLevel<P, L, NB, 0, 0>::run(cnt, p, word, nullptr, cq);  // weight 1024
          constexpr int LQ = BitsLevels<NB>::kQuad;
          if (i == 0 || i == 2) {
            pw[p] = cq;
          } else if (i == 1) {
            csa(cnt.A[p][LQ], pw[p], cq, pa[p]);
          } else {
            uint32_t pb;
            csa(cnt.A[p][LQ], pw[p], cq, pb);
            csa(cnt.A[p][LQ + 1], pa[p], pb, cmid[m][p]);
          }
        }
        continue;
      }
      // one word position at a time: 4 channels x NB planes live, not x P
      uint32_t carry[NB][4];  // consecutive words: the previous position's high word
#pragma unroll
      for (int p = 0; p < P; ++p) {
        uint32_t x[NB][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
#pragma unroll
          for (int b = 0; b < NB; ++b) {
            uint32_t lo = 0u, hi = 0u;
            if (live[q]) {
              if constexpr (BitsWords<P>::kContig) {
                lo = p == 0 ? base[q][b * slot_w] : carry[b][q];
                hi = base[q][b * slot_w + p + 1];
                carry[b][q] = hi;
              } else {
                lo = base[q][b * slot_w + 32 * p];
                hi = base[q][b * slot_w + 32 * p + 1];
              }
            }
            x[b][q] = __funnelshift_r(lo, hi, sh[q]);
          }
        }
        uint32_t cq;
        if constexpr (NB == 4) {
          cnt.quad4(p, x, cq);       // weight 64
        } else if constexpr (NB == 2) {
          const uint32_t lo[4] = {x[0][0], x[0][1], x[0][2], x[0][3]};
          const uint32_t hi[4] = {x[NB - 1][0], x[NB - 1][1], x[NB - 1][2], x[NB - 1][3]};
          cnt.quad2(p, lo, hi, cq);  // weight 16
        } else {
          const uint32_t v[4] = {x[0][0], x[0][1], x[0][2], x[0][3]};
          cnt.quad1(p, v, cq);       // weight 4
        }
        constexpr int LQ = BitsLevels<NB>::kQuad;  // level of the per-quad carries
        if (i == 0 || i == 2) {
          pw[p] = cq;
        } else if (i == 1) {
          csa(cnt.A[p][LQ], pw[p], cq, pa[p]);
        } else {
          uint32_t pb;
          csa(cnt.A[p][LQ], pw[p], cq, pb);
          csa(cnt.A[p][LQ + 1], pa[p], pb, cmid[m][p]);  // weight 64 (2-bit) / 16 (1-bit)
        }
      }
    }
  }
  constexpr int LM = BitsLevels<NB>::kQuad + 2;  // level of the per-16-channel carries
#pragma unroll
  for (int p = 0; p < P; ++p) {
    if constexpr (NMID == 4) {
      const uint32_t w4[4] = {cmid[0][p], cmid[1][p], cmid[2][p], cmid[3][p]};
      uint32_t top;
      cnt.fold4(p, LM, w4, top);
      cnt.ripple(p, LM + 2, top);
    } else if constexpr (NMID == 1) {
      cnt.ripple(p, LM, cmid[0][p]);
    } else {
      uint32_t top;
      csa(cnt.A[p][LM], cmid[0][p], cmid[1][p], top);
      cnt.ripple(p, LM + 1, top);
    }
  }
}

template <int P, int L>
__device__ __forceinline__ void store_bits_counts(const BitCounter<P, L>& cnt, const DmtArgs& a,
                                                  int dm, int64_t t0, int wbase);

template <int NB, int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT>
__device__ __forceinline__ void dmt_bits_body(const DmtArgs& a) {
  using Sh = BitsShape<NB, P, DW, TW, SLAB>;
  constexpr int NWC = Sh::kNwc;
  constexpr int T = Sh::kT;
  constexpr int JJ = (SLAB + 31) / 32;
  static_assert(SLAB == 16 || SLAB == 32 || SLAB == 64, "slab of 16, 32 or 64 channels");

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* sdata = reinterpret_cast<uint32_t*>(smem);
  int2* soff = reinterpret_cast<int2*>(sdata + (int64_t)STAGES * SLAB * NB * a.slot_w);
  uint64_t* full = reinterpret_cast<uint64_t*>(soff + STAGES * DW * SLAB);
  uint64_t* empty = full + STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int dm0 = blockIdx.x * DW;
  const int64_t t0 = (int64_t)blockIdx.y * T;
  const int nslab = (a.nchans + SLAB - 1) / SLAB;

  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NWC);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NWC) {
    // producer: delays -> staged window start (16-B aligned word) and each DM
    // row's sample offset within the staged window
    const uint32_t* planar = static_cast<const uint32_t*>(a.planar);
    for (int k = 0; k < nslab; ++k) {
      const int s = k % STAGES;
      const int c0 = k * SLAB;
      const int nc = min(SLAB, a.nchans - c0);
      int32_t dv[JJ][DW];
      int32_t mn[JJ], mx[JJ];
      // the delay loads do not depend on the slot: issue them before waiting
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj) {
        const int j = lane + jj * 32;
        mn[jj] = INT32_MAX;
        mx[jj] = INT32_MIN;
#pragma unroll
        for (int i = 0; i < DW; ++i) {
          int32_t d = 0;
          if (j < nc) {
            const int dm = min(dm0 + i, a.ndm - 1);
            d = a.sign * __ldg(a.delays + (int64_t)dm * a.dpitch + c0 + j);
            if (d < a.dlo || d > a.dhi) {
              dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)(c0 + j));
              d = min(max(d, a.dlo), a.dhi);
            }
          }
          dv[jj][i] = d;
          mn[jj] = min(mn[jj], d);
          mx[jj] = max(mx[jj], d);
        }
      }
      if (k >= STAGES && !mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, a.status)) break;
      int64_t ws_reg[JJ];
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj) {
        const int j = lane + jj * 32;
        ws_reg[jj] = 0;
        if (j < nc) {
          if (mx[jj] - mn[jj] > a.span_max) {
            dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)(c0 + j) | 0x80000000u);
            mx[jj] = mn[jj] + a.span_max;
          }
          const int64_t ws = ((t0 + mn[jj] + a.halo) / 32) & ~int64_t(3);
          const int32_t base = (int32_t)(ws * 32 - a.halo - t0);
#pragma unroll
          for (int i = 0; i < DW; ++i) {
            const int32_t o = min(dv[jj][i], mx[jj]) - base;  // >= 0: base <= min delay
            soff[(s * DW + i) * SLAB + j] = make_int2(o >> 5, o & 31);
          }
          ws_reg[jj] = ws;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive_expect_tx(&full[s], (uint32_t)nc * NB * a.slot_w * 4u);
      __syncwarp();
#pragma unroll
      for (int jj = 0; jj < JJ; ++jj) {
        const int j = lane + jj * 32;
        if (j < nc) {
#pragma unroll
          for (int b = 0; b < NB; ++b)
            bulk_g2s(sdata + (((int64_t)s * SLAB + j) * NB + b) * a.slot_w,
                     planar + ((int64_t)(c0 + j) * NB + b) * a.pitch_w + ws_reg[jj],
                     a.slot_w * 4u, &full[s]);
        }
      }
    }
    return;
  }

  // consumers: warp (dmw, tw); thread words w = wbase + BitsWords<P>::pos(p)
  const int dmw = warp / TW, tw = warp % TW;
  const int dm = dm0 + dmw;
  const int wbase = BitsWords<P>::base(tw, lane);
  BitCounter<P, L> cnt;
  cnt.zero();
  bool ok = true;
  for (int k = 0; k < nslab; ++k) {
    const int s = k % STAGES;
    if (!mbar_wait(&full[s], (k / STAGES) & 1, a.status)) { ok = false; break; }
    const int nc = min(SLAB, a.nchans - k * SLAB);
    const uint32_t* sd = sdata + (int64_t)s * SLAB * NB * a.slot_w;
    const int2* off = soff + (s * DW + dmw) * SLAB;
    if (nc == SLAB) bits_slab<NB, P, L, SLAB, true, SLOT>(cnt, sd, off, nc, a.slot_w, wbase);
    else bits_slab<NB, P, L, SLAB, false, SLOT>(cnt, sd, off, nc, a.slot_w, wbase);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok || dm >= a.ndm) return;
  store_bits_counts<P, L>(cnt, a, dm, t0, wbase);
}

// Counts of DM row dm: word p covers samples t0 + 32*(wbase + pos(p)) + i.
template <int P, int L>
__device__ __forceinline__ void store_bits_counts(const BitCounter<P, L>& cnt, const DmtArgs& a,
                                                  int dm, int64_t t0, int wbase) {
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int64_t tb = t0 + 32LL * (wbase + BitsWords<P>::pos(p));
    if (a.out_kind == SPP_OUT_I32) {
      int32_t* out = static_cast<int32_t*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
      if (tb + 32 <= a.nvalid && ((reinterpret_cast<uintptr_t>(out + tb) & 15) == 0)) {
#pragma unroll
        for (int i = 0; i < 32; i += 4) {
          int4 v;
          v.x = (int)cnt.count(p, i);
          v.y = (int)cnt.count(p, i + 1);
          v.z = (int)cnt.count(p, i + 2);
          v.w = (int)cnt.count(p, i + 3);
          *reinterpret_cast<int4*>(out + tb + i) = v;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (tb + i < a.nvalid) out[tb + i] = (int32_t)cnt.count(p, i);
      }
    } else if (a.out_kind == SPP_OUT_U16) {
      uint16_t* out = static_cast<uint16_t*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (tb + i < a.nvalid) out[tb + i] = (uint16_t)min(cnt.count(p, i), 65535u);
    } else {
      float* out = static_cast<float*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (tb + i < a.nvalid) out[tb + i] = (float)cnt.count(p, i);
    }
  }
}

// The kernel without a minimum-residency hint (ptxas picks the register
// count), and the same body with one (registers capped for MINB CTAs per SM).
template <int NB, int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT = 0>
__global__ void __launch_bounds__(BitsShape<NB, P, DW, TW, SLAB>::kThreads)
k_dmt_bits(const DmtArgs a) {
  dmt_bits_body<NB, P, DW, TW, STAGES, L, SLAB, SLOT>(a);
}
template <int NB, int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT, int MINB>
__global__ void __launch_bounds__(BitsShape<NB, P, DW, TW, SLAB>::kThreads, MINB)
k_dmt_bits_minb(const DmtArgs a) {
  dmt_bits_body<NB, P, DW, TW, STAGES, L, SLAB, SLOT>(a);
}

// 32 x 32 bit transpose across a warp: lane j holds row j (bit i = column
// i); afterwards lane i holds column i (bit j = row j).  Five rounds, each
// swapping the off-diagonal s x s blocks with the lane s apart.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const uint32_t m = s == 16 ? 0x0000FFFFu : s == 8 ? 0x00FF00FFu : s == 4 ? 0x0F0F0F0Fu
                     : s == 2 ? 0x33333333u : 0x55555555u;  // bits whose index has bit s clear
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, s);
    const bool up = (lane & s) != 0;
    const uint32_t t = up ? (y >> s) : (y << s);
    const uint32_t keep = up ? ~m : m;
    x = (x & keep) | (t & ~keep);
  }
  return x;
}

// Corner turn into bit-plane rows (row c*NB + b: bit b of channel c, 32
// samples per word).  CTA = planes_ct_chans(NB) channels x kPlaneWords words
// (256 raw rows).
template <int NB>
__global__ void __launch_bounds__(256)
k_corner_turn_planes(const uint8_t* __restrict__ raw, int64_t nchans, int64_t nsamps,
                     int bitorder, int64_t halo, uint32_t* __restrict__ planar,
                     int64_t pitch_w) {
  constexpr int CC = planes_ct_chans(NB);
  constexpr int RT = kPlaneWords * 32;
  constexpr int SB = CC * NB / 8;
  constexpr int SBP = SB + 4;
  __shared__ __align__(16) uint8_t s_raw[RT * SBP];
  __shared__ uint32_t s_out[CC * NB][kPlaneWords + 1];
  const int64_t c0 = (int64_t)blockIdx.x * CC;
  const int nc = (int)((nchans - c0) < CC ? (nchans - c0) : CC);
  const int seg = (nc * NB + 7) / 8;
  const int64_t rowbytes = nchans * NB / 8;
  const int64_t segstart = c0 * NB / 8;
  const bool vec = ((rowbytes & 3) == 0) && ((segstart & 3) == 0) && ((seg & 3) == 0) &&
                   ((reinterpret_cast<uintptr_t>(raw) & 3) == 0);
  const bool vec16 = ((rowbytes & 15) == 0) && ((segstart & 15) == 0) && ((seg & 15) == 0) &&
                     ((reinterpret_cast<uintptr_t>(raw) & 15) == 0);
  // plane words leave in 16-byte stores (pitches are multiples of 4 words and
  // tiles start at multiples of 8)
  const bool st16 = ((pitch_w & 3) == 0) && ((reinterpret_cast<uintptr_t>(planar) & 15) == 0);
  const int64_t ntw = (pitch_w + kPlaneWords - 1) / kPlaneWords;
  for (int64_t by = blockIdx.y; by < ntw; by += gridDim.y) {
    const int64_t w0 = by * kPlaneWords;
    if (vec16) {
      const int nq = seg >> 4;
      for (int idx = threadIdx.x; idx < RT * nq; idx += blockDim.x) {
        const int r = idx / nq, k = idx - r * nq;
        const int64_t row = wrap_row(w0 * 32 + r - halo, nsamps);
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (row >= 0) v = __ldg(reinterpret_cast<const uint4*>(raw + row * rowbytes + segstart) + k);
        uint32_t* d = reinterpret_cast<uint32_t*>(s_raw + r * SBP + 16 * k);
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
        d[3] = v.w;
      }
    } else if (vec) {
      const int nw = seg >> 2;
      for (int idx = threadIdx.x; idx < RT * nw; idx += blockDim.x) {
        const int r = idx / nw, k = idx - r * nw;
        const int64_t row = wrap_row(w0 * 32 + r - halo, nsamps);
        uint32_t v = 0;
        if (row >= 0) v = __ldg(reinterpret_cast<const uint32_t*>(raw + row * rowbytes + segstart) + k);
        *reinterpret_cast<uint32_t*>(s_raw + r * SBP + 4 * k) = v;
      }
    } else {
      for (int idx = threadIdx.x; idx < RT * seg; idx += blockDim.x) {
        const int r = idx / seg, k = idx - r * seg;
        const int64_t row = wrap_row(w0 * 32 + r - halo, nsamps);
        s_raw[r * SBP + k] = (row >= 0) ? __ldg(raw + row * rowbytes + segstart + k) : 0;
      }
    }
    __syncthreads();
    // one warp per (word w, 4-byte column group g): lane j loads the group's
    // 32 bits of row 32w + j, a 32 x 32 bit transpose leaves in lane i bit i
    // of all 32 rows -- the plane word (32 samples, LSB first) of the
    // (channel, plane) that bit i of the packed bytes holds
    {
      constexpr int NG = SB / 4;  // column groups per row segment
      const int lane = threadIdx.x & 31;
      const int bi = lane >> 3, bb = lane & 7;
      const int q = (bitorder == SPP_BITORDER_BIG) ? (7 - bb) / NB : bb / NB;
      for (int task = threadIdx.x >> 5; task < kPlaneWords * NG; task += blockDim.x >> 5) {
        const int w = task / NG, g = task - w * NG;
        uint32_t x = *reinterpret_cast<const uint32_t*>(s_raw + (w * 32 + lane) * SBP + 4 * g);
        x = warp_transpose32(x, lane);
        const int c = (4 * g + bi) * (8 / NB) + q;
        s_out[c * NB + bb % NB][w] = x;
      }
    }
    __syncthreads();
    if (st16) {
      for (int idx = threadIdx.x; idx < CC * NB * (kPlaneWords / 4); idx += blockDim.x) {
        const int w = 4 * (idx % (kPlaneWords / 4)), rr = idx / (kPlaneWords / 4);
        if (rr < nc * NB && w0 + w < pitch_w)
          *reinterpret_cast<uint4*>(planar + (c0 * NB + rr) * pitch_w + w0 + w) =
              make_uint4(s_out[rr][w], s_out[rr][w + 1], s_out[rr][w + 2], s_out[rr][w + 3]);
      }
    } else {
      for (int idx = threadIdx.x; idx < CC * NB * kPlaneWords; idx += blockDim.x) {
        const int w = idx % kPlaneWords, rr = idx / kPlaneWords;
        if (rr < nc * NB && w0 + w < pitch_w) planar[(c0 * NB + rr) * pitch_w + w0 + w] = s_out[rr][w];
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------
// Channel-pair sums of 2-bit data.
//
// The transform's sum over channels is regrouped into pairs (2k, 2k+1):
//   out[dm][t] = sum_k S_k,r[t + o(dm, 2k)],   S_k,r[t] = x[2k][t] + x[2k+1][t + r]
// with r = o(dm, 2k+1) - o(dm, 2k).  Over a DM grid each pair sees few
// distinct r (the delay difference of two adjacent channels), so every
// (pair, r) row is summed once and shared by all DMs that use it: the DM
// kernel then adds 3 bit planes per two channels instead of 4 -- the same
// integers in another order, so the sums are exact.
// ----------------------------------------------------------------------------

// Pair-sum rows: row i = (pair k, offset r) = src[i]; its planes b = 0..2 are
// rows 3i + b of `out` on the channel rows' grid (same halo and pitch).  Each
// thread makes four consecutive words; partner words outside channel 2k+1's
// row read as zero (such words feed no valid output).
static __global__ void __launch_bounds__(256)
k_pair_sums2(const uint32_t* __restrict__ planar, int64_t pitch_w, const int2* __restrict__ src,
             uint32_t* __restrict__ out) {
  const int64_t row = blockIdx.x;
  const int2 kr = __ldg(src + row);
  const int64_t w = ((int64_t)blockIdx.y * blockDim.x + threadIdx.x) * 4;
  if (w >= pitch_w) return;
  const uint32_t* a0 = planar + (int64_t)(2 * kr.x) * 2 * pitch_w;   // channel 2k, plane 0
  const uint32_t* b0 = a0 + 2 * pitch_w;                              // channel 2k+1, plane 0
  const int q = kr.y >> 5, s = kr.y & 31;                             // floor(r / 32), r mod 32
  const uint4 al = *reinterpret_cast<const uint4*>(a0 + w);
  const uint4 ah = *reinterpret_cast<const uint4*>(a0 + pitch_w + w);
  uint32_t bl[5], bh[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int64_t j = w + q + i;
    const bool in = j >= 0 && j < pitch_w;
    bl[i] = in ? __ldg(b0 + j) : 0u;
    bh[i] = in ? __ldg(b0 + pitch_w + j) : 0u;
  }
  const uint32_t xl[4] = {al.x, al.y, al.z, al.w}, xh[4] = {ah.x, ah.y, ah.z, ah.w};
  uint32_t s0[4], s1[4], s2[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t yl = __funnelshift_r(bl[i], bl[i + 1], s);
    const uint32_t yh = __funnelshift_r(bh[i], bh[i + 1], s);
    const uint32_t c0 = xl[i] & yl;  // x + y, two 2-bit numbers: ripple add
    s0[i] = xl[i] ^ yl;
    s1[i] = xh[i] ^ yh ^ c0;
    s2[i] = (xh[i] & yh) | (xh[i] & c0) | (yh & c0);
  }
  uint32_t* o = out + row * 3 * pitch_w + w;
  *reinterpret_cast<uint4*>(o) = make_uint4(s0[0], s0[1], s0[2], s0[3]);
  *reinterpret_cast<uint4*>(o + pitch_w) = make_uint4(s1[0], s1[1], s1[2], s1[3]);
  *reinterpret_cast<uint4*>(o + 2 * pitch_w) = make_uint4(s2[0], s2[1], s2[2], s2[3]);
}

// Shared memory per stage of the pair kernel: SLAB pairs x 2 staged rows x 3
// planes x slot_w words, plus DW x SLAB decoded offsets.
__host__ __device__ constexpr int64_t pair_stage_bytes(int slab, int slot_w, int dw) {
  return (int64_t)slab * 2 * 3 * slot_w * 4 + (int64_t)dw * slab * 8;
}

// The pair kernel keeps counter levels below kPairRegLevels in registers;
// the upper levels, which change only when a carry ripples up (once per two
// slabs), live in a per-thread slice of shared memory.
constexpr int kPairRegLevels = 8;
__host__ __device__ constexpr int64_t pair_hi_bytes(int p, int nwc) {
  return (int64_t)(BitsLevels<3>::kLevels - kPairRegLevels) * p * nwc * 32 * 4;
}

// Level of the one carry word a slab of SLAB pairs leaves (quad carries of
// weight 32 folded pairwise).
template <int SLAB>
__host__ __device__ constexpr int pairs_top_level() {
  return BitsLevels<3>::kQuad + (SLAB == 8 ? 1 : SLAB == 16 ? 2 : 3);
}

// One slab of SLAB pairs (SLAB = 8, 16 or 32) through the counter: quads of
// pairs through the three-plane network (carry of weight 32), their carries
// folded pairwise; the slab's single carry (level pairs_top_level<SLAB>) is
// returned in top[] for the caller to fold with the next slab's.  off[j]
// holds the staged row's start word (row included) and the bit shift.
template <int P, int L, int SLAB, bool FULL>
__device__ __forceinline__ void pairs_slab(BitCounter<P, L>& cnt, const uint32_t* __restrict__ sd,
                                           const int2* __restrict__ off, int nc, int slot_w,
                                           int wbase, uint32_t (&top)[P]) {
  static_assert(SLAB == 8 || SLAB == 16 || SLAB == 32, "slab of 8, 16 or 32 pairs");
  constexpr int NQ = SLAB / 4;
  constexpr int LQ = BitsLevels<3>::kQuad;
  uint32_t pw[P], pa[P], cm[2][P];
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    const uint32_t* base[4];
    int sh[4];
    bool live[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = 4 * i + q;
      live[q] = FULL || j < nc;
      const int2 ow = live[q] ? off[j] : make_int2(0, 0);
      sh[q] = ow.y;
      base[q] = sd + ow.x + wbase;
    }
    uint32_t carry[3][4];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      uint32_t x[3][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          uint32_t lo = 0u, hi = 0u;
          if (live[q]) {
            if constexpr (BitsWords<P>::kContig) {
              lo = p == 0 ? base[q][b * slot_w] : carry[b][q];
              hi = base[q][b * slot_w + p + 1];
              carry[b][q] = hi;
            } else {
              lo = base[q][b * slot_w + 32 * p];
              hi = base[q][b * slot_w + 32 * p + 1];
            }
          }
          x[b][q] = __funnelshift_r(lo, hi, sh[q]);
        }
      }
      auto word = [&](int b, int q) -> uint32_t { return x[b][q]; };
      uint32_t cq;
      QuadLevel<P, L, 3, 0, 0>::run(cnt, p, word, nullptr, cq);  // weight 32
      if constexpr (NQ == 2) {
        if (i == 0) pw[p] = cq;
        else csa(cnt.A[p][LQ], pw[p], cq, top[p]);  // weight 64
      } else {
        const int m = i / 4;  // group of four quads (16 pairs)
        if (i % 4 == 0 || i % 4 == 2) {
          pw[p] = cq;
        } else if (i % 4 == 1) {
          csa(cnt.A[p][LQ], pw[p], cq, pa[p]);
        } else {
          uint32_t pb;
          csa(cnt.A[p][LQ], pw[p], cq, pb);
          csa(cnt.A[p][LQ + 1], pa[p], pb, cm[m][p]);  // weight 128
        }
      }
    }
  }
  if constexpr (NQ == 4) {
#pragma unroll
    for (int p = 0; p < P; ++p) top[p] = cm[0][p];
  } else if constexpr (NQ == 8) {
#pragma unroll
    for (int p = 0; p < P; ++p) csa(cnt.A[p][LQ + 2], cm[0][p], cm[1][p], top[p]);
  }
}

// DM-time transform over pair-sum rows.  CTA = DW DMs x one time tile, as
// the bit-sliced kernel; a slab is SLAB pairs.  The DW DMs read one to three
// distinct rows of a pair, 2 x SLAB rows per slab at most (the plan admits
// the kernel only for tables where that holds).  Time tiles are multiples of
// 128 samples, so where each DM reads within the staged windows does not
// depend on the tile: the plan precomputes it per (DM tile, slab), and the
// producer only issues bulk copies -- the offsets block and up to 2 x SLAB
// rows of three planes.
template <int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT>
__device__ __forceinline__ void dmt_pairs_body(const DmtArgs& a) {
  using Sh = BitsShape<3, P, DW, TW, SLAB>;
  constexpr int NWC = Sh::kNwc;
  constexpr int T = Sh::kT;
  static_assert(2 * SLAB <= 32, "one producer lane per staged row");
  static_assert(T % 128 == 0, "tile-independent staging needs 128-sample tiles");

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* sdata = reinterpret_cast<uint32_t*>(smem);
  int2* soff = reinterpret_cast<int2*>(sdata + (int64_t)STAGES * SLAB * 6 * a.slot_w);
  uint64_t* full = reinterpret_cast<uint64_t*>(soff + STAGES * DW * SLAB);
  uint64_t* empty = full + STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int dm0 = blockIdx.x * DW;
  const int64_t t0 = (int64_t)blockIdx.y * T;
  const int nslab = (a.npairs + SLAB - 1) / SLAB;

  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NWC);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NWC) {
    // producer: lane e stages row entry e of the slab
    const uint32_t* planar = static_cast<const uint32_t*>(a.planar);
    const int2* toff = a.pair_off + (int64_t)blockIdx.x * nslab * DW * SLAB;
    const int2* tent = a.pair_ent + (int64_t)blockIdx.x * nslab * 2 * SLAB;
    const int64_t tw0 = t0 / 32;
    for (int k = 0; k < nslab; ++k) {
      const int s = k % STAGES;
      const int2 en = lane < 2 * SLAB ? __ldg(tent + (int64_t)k * 2 * SLAB + lane) : make_int2(-1, 0);
      if (k >= STAGES && !mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, a.status)) break;
      const uint32_t nrow = __popc(__ballot_sync(0xffffffffu, en.x >= 0));
      if (lane == 0)
        mbar_arrive_expect_tx(&full[s], (uint32_t)(DW * SLAB * 8) + nrow * 3u * (uint32_t)a.slot_w * 4u);
      __syncwarp();
      if (lane == 0)
        bulk_g2s(soff + s * DW * SLAB, toff + (int64_t)k * DW * SLAB, DW * SLAB * 8, &full[s]);
      if (en.x >= 0) {
#pragma unroll
        for (int b = 0; b < 3; ++b)
          bulk_g2s(sdata + (((int64_t)s * 2 * SLAB + lane) * 3 + b) * a.slot_w,
                   planar + ((int64_t)en.x * 3 + b) * a.pitch_w + tw0 + en.y, a.slot_w * 4u,
                   &full[s]);
      }
    }
    return;
  }

  // consumers: warp (dmw, tw); thread words w = wbase + BitsWords<P>::pos(p)
  const int dmw = warp / TW, tw = warp % TW;
  const int dm = dm0 + dmw;
  const int wbase = BitsWords<P>::base(tw, lane);
  // levels [0, LR) in registers, [LR, L) in this thread's shared slice
  // (index ((l - LR) * P + p) * threads + thread: conflict-free)
  constexpr int LR = kPairRegLevels;
  static_assert(L > LR && pairs_top_level<SLAB>() < LR, "split counter levels");
  uint32_t* shi = reinterpret_cast<uint32_t*>(empty + STAGES);
  const int ct = threadIdx.x;
  auto hi = [&](int l, int p) -> uint32_t& { return shi[((l - LR) * P + p) * (NWC * 32) + ct]; };
#pragma unroll
  for (int l = LR; l < L; ++l)
#pragma unroll
    for (int p = 0; p < P; ++p) hi(l, p) = 0u;
  BitCounter<P, LR> cnt;
  cnt.zero();
  // carry word c of weight 2^l0 up through the register and shared levels
  auto ripple = [&](int p, int l0, uint32_t c) {
#pragma unroll
    for (int l = 0; l < LR; ++l) {
      if (l < l0) continue;
      uint32_t nc;
      half(cnt.A[p][l], c, nc);
      c = nc;
    }
#pragma unroll
    for (int l = LR; l < L; ++l) {
      if (c == 0u) break;
      uint32_t& h = hi(l, p);
      const uint32_t nc = h & c;
      h ^= c;
      c = nc;
    }
  };
  // slab carries are folded in pairs before they ripple up: one ripple per
  // two slabs
  constexpr int LT = pairs_top_level<SLAB>();
  uint32_t hold[P];
  bool ok = true;
  for (int k = 0; k < nslab; ++k) {
    const int s = k % STAGES;
    if (!mbar_wait(&full[s], (k / STAGES) & 1, a.status)) { ok = false; break; }
    const int nc = min(SLAB, a.npairs - k * SLAB);
    const uint32_t* sd = sdata + (int64_t)s * SLAB * 6 * a.slot_w;
    const int2* off = soff + (s * DW + dmw) * SLAB;
    const int slot_w = SLOT > 0 ? SLOT : a.slot_w;
    uint32_t top[P];
    if (nc == SLAB) pairs_slab<P, LR, SLAB, true>(cnt, sd, off, nc, slot_w, wbase, top);
    else pairs_slab<P, LR, SLAB, false>(cnt, sd, off, nc, slot_w, wbase, top);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (k & 1) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        uint32_t c;
        csa(cnt.A[p][LT], hold[p], top[p], c);
        ripple(p, LT + 1, c);
      }
    } else {
#pragma unroll
      for (int p = 0; p < P; ++p) hold[p] = top[p];
    }
  }
  if (!ok || dm >= a.ndm) return;
  if (nslab & 1) {
#pragma unroll
    for (int p = 0; p < P; ++p) ripple(p, LT, hold[p]);
  }
  BitCounter<P, L> all;
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int l = 0; l < L; ++l) all.A[p][l] = l < LR ? cnt.A[p][l] : hi(l, p);
  }
  store_bits_counts<P, L>(all, a, dm, t0, wbase);
}

template <int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT = 0>
__global__ void __launch_bounds__(BitsShape<3, P, DW, TW, SLAB>::kThreads)
k_dmt_pairs(const DmtArgs a) {
  dmt_pairs_body<P, DW, TW, STAGES, L, SLAB, SLOT>(a);
}
template <int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT, int MINB>
__global__ void __launch_bounds__(BitsShape<3, P, DW, TW, SLAB>::kThreads, MINB)
k_dmt_pairs_minb(const DmtArgs a) {
  dmt_pairs_body<P, DW, TW, STAGES, L, SLAB, SLOT>(a);
}
// k_dmt_wl; planar rows are bit-plane rows, NB per channel).
// ----------------------------------------------------------------------------
template <int NB, int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT>
__device__ __forceinline__ void dmt_bits_wl_body(const WlArgs& w) {
  using Sh = BitsShape<NB, P, DW, TW, SLAB>;
  constexpr int NWC = Sh::kNwc;
  constexpr int JJ = (SLAB + 31) / 32;

  extern __shared__ __align__(128) unsigned char smem[];
  uint32_t* sdata = reinterpret_cast<uint32_t*>(smem);
  int2* soff = reinterpret_cast<int2*>(sdata + (int64_t)STAGES * SLAB * NB * w.slot_w);
  int32_t* stag = reinterpret_cast<int32_t*>(soff + STAGES * DW * SLAB);  // per stage: item, slab, nslab, pad
  uint64_t* full = reinterpret_cast<uint64_t*>(stag + 4 * STAGES);
  uint64_t* empty = full + STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NWC);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NWC) {
    uint32_t gk = 0;
    bool ok = true;
    while (ok) {
      int it_idx = 0;
      if (lane == 0) it_idx = atomicAdd(w.counter, 1);
      it_idx = __shfl_sync(0xffffffffu, it_idx, 0);
      if (it_idx >= w.nitems) break;
      const DmtItem it = w.items[it_idx];
      const uint32_t* planar = static_cast<const uint32_t*>(it.planar);
      const int nslab = (it.nchans + SLAB - 1) / SLAB;
      for (int k = 0; k < nslab; ++k, ++gk) {
        const int s = gk % STAGES;
        const int c0 = k * SLAB;
        const int nc = min(SLAB, it.nchans - c0);
        int32_t dv[JJ][DW];
        int32_t mn[JJ], mx[JJ];
#pragma unroll
        for (int jj = 0; jj < JJ; ++jj) {
          const int j = lane + jj * 32;
          mn[jj] = INT32_MAX;
          mx[jj] = INT32_MIN;
#pragma unroll
          for (int i = 0; i < DW; ++i) {
            int32_t d = 0;
            if (j < nc) {
              const int r = min(i, it.nrows - 1);
              d = it.sign * __ldg(it.delays + (int64_t)r * it.dpitch + c0 + j);
              if (d < it.dlo || d > it.dhi) {
                dev_flag(w.status, SPP_DEV_RANGE, (uint32_t)(c0 + j));
                d = min(max(d, it.dlo), it.dhi);
              }
            }
            dv[jj][i] = d;
            mn[jj] = min(mn[jj], d);
            mx[jj] = max(mx[jj], d);
          }
        }
        if (gk >= STAGES && !mbar_wait(&empty[s], ((gk / STAGES) - 1) & 1, w.status)) {
          ok = false;
          break;
        }
        int64_t ws_reg[JJ];
#pragma unroll
        for (int jj = 0; jj < JJ; ++jj) {
          const int j = lane + jj * 32;
          ws_reg[jj] = 0;
          if (j < nc) {
            if (mx[jj] - mn[jj] > it.span_max) {
              dev_flag(w.status, SPP_DEV_RANGE, (uint32_t)(c0 + j) | 0x80000000u);
              mx[jj] = mn[jj] + it.span_max;
            }
            const int64_t ws = ((it.t0 + mn[jj] + it.halo) / 32) & ~int64_t(3);
            const int32_t base = (int32_t)(ws * 32 - it.halo - it.t0);
#pragma unroll
            for (int i = 0; i < DW; ++i) {
              const int32_t o = min(dv[jj][i], mx[jj]) - base;  // >= 0: base <= min delay
              soff[(s * DW + i) * SLAB + j] = make_int2(o >> 5, o & 31);
            }
            ws_reg[jj] = ws;
          }
        }
        if (lane == 0) {
          stag[4 * s + 0] = it_idx;
          stag[4 * s + 1] = k;
          stag[4 * s + 2] = nslab;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&full[s], (uint32_t)nc * NB * w.slot_w * 4u);
        __syncwarp();
#pragma unroll
        for (int jj = 0; jj < JJ; ++jj) {
          const int j = lane + jj * 32;
          if (j < nc) {
#pragma unroll
            for (int b = 0; b < NB; ++b)
              bulk_g2s(sdata + (((int64_t)s * SLAB + j) * NB + b) * w.slot_w,
                       planar + ((int64_t)(c0 + j) * NB + b) * it.pitch_w + ws_reg[jj],
                       w.slot_w * 4u, &full[s]);
          }
        }
      }
    }
    if (ok) {
      const int s = gk % STAGES;
      if (gk < STAGES || mbar_wait(&empty[s], ((gk / STAGES) - 1) & 1, w.status)) {
        if (lane == 0) {
          stag[4 * s + 0] = -1;
          mbar_arrive(&full[s]);
        }
      }
    }
    return;
  }

  const int dmw = warp / TW, tw = warp % TW;
  const int wbase = BitsWords<P>::base(tw, lane);
  BitCounter<P, L> cnt;
  cnt.zero();
  DmtItem it{};
  for (uint32_t gk = 0;; ++gk) {
    const int s = gk % STAGES;
    if (!mbar_wait(&full[s], (gk / STAGES) & 1, w.status)) return;
    const int it_idx = stag[4 * s + 0];
    if (it_idx < 0) return;
    const int k = stag[4 * s + 1], nslab = stag[4 * s + 2];
    if (k == 0) {
      it = w.items[it_idx];
      cnt.zero();
    }
    const int nc = min(SLAB, it.nchans - k * SLAB);
    const uint32_t* sd = sdata + (int64_t)s * SLAB * NB * w.slot_w;
    const int2* off = soff + (s * DW + dmw) * SLAB;
    if (nc == SLAB) bits_slab<NB, P, L, SLAB, true, SLOT>(cnt, sd, off, nc, w.slot_w, wbase);
    else bits_slab<NB, P, L, SLAB, false, SLOT>(cnt, sd, off, nc, w.slot_w, wbase);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (k == nslab - 1 && dmw < it.nrows) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const int64_t tb = it.t0 + 32LL * (wbase + BitsWords<P>::pos(p));
        if (it.out_kind == SPP_OUT_I32) {
          int32_t* out = static_cast<int32_t*>(it.out) + (int64_t)dmw * it.out_stride + it.out_start;
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (tb + i < it.nvalid) out[tb + i] = (int32_t)cnt.count(p, i);
        } else if (it.out_kind == SPP_OUT_U16) {
          uint16_t* out = static_cast<uint16_t*>(it.out) + (int64_t)dmw * it.out_stride + it.out_start;
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (tb + i < it.nvalid) out[tb + i] = (uint16_t)min(cnt.count(p, i), 65535u);
        } else {
          float* out = static_cast<float*>(it.out) + (int64_t)dmw * it.out_stride + it.out_start;
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (tb + i < it.nvalid) out[tb + i] = (float)cnt.count(p, i);
        }
      }
    }
  }
}

// Work-list kernel without / with a minimum-residency hint (SLOT > 0: the
// launch's slot width must equal SLOT).
template <int NB, int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT = 0>
__global__ void __launch_bounds__(BitsShape<NB, P, DW, TW, SLAB>::kThreads)
k_dmt_bits_wl(const WlArgs w) {
  dmt_bits_wl_body<NB, P, DW, TW, STAGES, L, SLAB, SLOT>(w);
}
template <int NB, int P, int DW, int TW, int STAGES, int L, int SLAB, int SLOT, int MINB>
__global__ void __launch_bounds__(BitsShape<NB, P, DW, TW, SLAB>::kThreads, MINB)
k_dmt_bits_wl_minb(const WlArgs w) {
  dmt_bits_wl_body<NB, P, DW, TW, STAGES, L, SLAB, SLOT>(w);
}
}  // namespace spp
