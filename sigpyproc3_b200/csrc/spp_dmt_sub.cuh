// Float64 DM-time transform of float32 rows with shared channel-group sums.
//
// The brute-force float64 kernel (k_dmt<32, ..., SPP_ACC_F64>) converts every
// staged float32 sample to float64 for every trial that reads it, and that
// conversion is its limit.  Within a tile of DW adjacent trials, the delays of
// a group of four adjacent channels mostly differ from trial to trial by a
// common shift: d_i(4g + j) = d_i(4g) + r(j) with the same residuals r for many
// trials.  Each distinct residual pattern of a group ("pattern") gets one row
// of float64 partial sums
//     P[tau] = sum_j x[4g + j][bmin + r(j) + tau],  tau < T + bspan,
// (stage 1), and each trial adds the row of its pattern at its own shift,
//     out_i[t] += P[d_i(4g) - bmin + t]              (stage 2),
// which is the same sum  sum_j x[4g + j][t + d_i(4g + j)]  with one float64
// load per four channels instead of four conversions.  The sums are float64
// throughout, in channel order within a group and group order across groups:
// equal to the channel-ordered float64 sum of the reference loop whenever no
// partial sum rounds (float32 inputs within a 2^26 dynamic range), and within
// one float64 rounding per group otherwise.
//
// The patterns of each (DM tile, group) are found on the host when the plan is
// made (spp_core.cu) and stored as records that the producer warp stages with
// the slab's rows:
//   int32 [0] npat, [1..3] unused,
//         [4 .. 4 + DW)       per trial: (pattern << 16) | (d_i(4g) - bmin)
//         [4 + DW + 5 k ...]  per pattern k: r1, r2, r3, bmin, bspan
// The consumers meet at two mbarriers per slab (partial rows written; partial
// rows read), each wait bounded like every other wait in the library.
#pragma once

#include "spp_dmt.cuh"

namespace spp {

constexpr int kSubGroup = 4;  // channels per group

__host__ __device__ constexpr int sub_rec_words(int dw) { return 4 + 6 * dw; }

// Bytes of one ring stage: the slab's staged rows, its channel window starts
// and its group records.
__host__ __device__ constexpr int64_t sub_stage_bytes(int slab, int slot_w, int dw) {
  return (int64_t)slab * slot_w * 4 + (int64_t)slab * 4 +
         (int64_t)(slab / kSubGroup) * sub_rec_words(dw) * 4;
}

template <int R, int DW, int TW, int SLAB, int STAGES>
__global__ void __launch_bounds__(DmtShape<32, R, DW, TW, SLAB, STAGES>::kThreads)
k_dmt_f64sub(const DmtArgs a) {
  using Sh = DmtShape<32, R, DW, TW, SLAB, STAGES>;
  constexpr int NWC = Sh::kNwc;
  constexpr int T = Sh::kT;
  constexpr int NG = SLAB / kSubGroup;
  constexpr int RW = sub_rec_words(DW);
  static_assert(SLAB % kSubGroup == 0 && SLAB <= 32, "slab of whole groups, one lane each");
  static_assert((RW * 4) % 16 == 0, "records must be whole 16-byte chunks");

  extern __shared__ __align__(128) unsigned char smem[];
  float* sraw = reinterpret_cast<float*>(smem);
  int32_t* swin = reinterpret_cast<int32_t*>(sraw + (int64_t)STAGES * SLAB * a.slot_w);
  int32_t* srec = swin + STAGES * SLAB;
  double* pbuf = reinterpret_cast<double*>(srec + STAGES * NG * RW);
  uint64_t* full = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(pbuf) + a.sub_pbytes);
  uint64_t* empty = full + STAGES;
  uint64_t* pbar = empty + STAGES;  // [0]: partial rows written, [1]: partial rows read

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
    mbar_init(&pbar[0], NWC);
    mbar_init(&pbar[1], NWC);
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == NWC) {
    // ---------------- producer warp: one lane per channel of the slab ----------------
    const float* planar = static_cast<const float*>(a.planar);
    for (int k = 0; k < nslab; ++k) {
      const int s = k % STAGES;
      const int c0 = k * SLAB;
      const int nc = min(SLAB, a.nchans - c0);
      int32_t mn = INT32_MAX, mx = INT32_MIN;
      if (lane < nc) {
#pragma unroll
        for (int i = 0; i < DW; ++i) {
          const int dm = min(dm0 + i, a.ndm - 1);
          int32_t d = __ldg(a.delays + (int64_t)dm * a.dpitch + c0 + lane);
          if (d < a.dlo || d > a.dhi) {
            dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)(c0 + lane));
            d = min(max(d, a.dlo), a.dhi);
          }
          mn = min(mn, d);
          mx = max(mx, d);
        }
      }
      if (k >= STAGES && !mbar_wait(&empty[s], ((k / STAGES) - 1) & 1, a.status)) break;
      int64_t ws = 0;
      if (lane < nc) {
        if (mx - mn > a.span_max) dev_flag(a.status, SPP_DEV_RANGE, (uint32_t)(c0 + lane) | 0x80000000u);
        ws = (t0 + mn + a.halo) & ~int64_t(3);  // 16-B aligned window start (words)
        swin[s * SLAB + lane] = (int32_t)(ws - a.halo - t0);
      }
      __syncwarp();
      const int ngc = nc / kSubGroup;
      if (lane == 0)
        mbar_arrive_expect_tx(&full[s], (uint32_t)nc * a.slot_w * 4u + (uint32_t)ngc * RW * 4u);
      __syncwarp();
      if (lane < nc)
        bulk_g2s(sraw + ((int64_t)s * SLAB + lane) * a.slot_w,
                 planar + (int64_t)(c0 + lane) * a.pitch_w + ws, a.slot_w * 4u, &full[s]);
      if (lane == 0)
        bulk_g2s(srec + s * NG * RW,
                 a.sub_tab + ((int64_t)blockIdx.x * a.sub_ngroups + c0 / kSubGroup) * RW,
                 (uint32_t)ngc * RW * 4u, &full[s]);
    }
    return;
  }

  // ---------------- consumer warps: (trial dmw, time part tw) ----------------
  const int dmw = warp / TW, tw = warp % TW;
  const int dm = dm0 + dmw;
  const int wbase = tw * 32 * R + lane;
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;
  bool ok = true;
  for (int k = 0; k < nslab; ++k) {
    const int s = k % STAGES;
    if (!mbar_wait(&full[s], (k / STAGES) & 1, a.status)) { ok = false; break; }
    const int nc = min(SLAB, a.nchans - k * SLAB);
    const int ng = nc / kSubGroup;
    const float* sd = sraw + (int64_t)s * SLAB * a.slot_w;
    const int32_t* win = swin + s * SLAB;
    const int32_t* rec = srec + s * NG * RW;
    // stage 1: partial rows, one warp per row in turn; rowbase[g] = first row of group g
    int rowbase[NG];
    {
      int row = 0;
      int64_t poff = 0;
#pragma unroll
      for (int gl = 0; gl < NG; ++gl) {
        rowbase[gl] = (int)poff;
        if (gl >= ng) continue;
        const int32_t* rg = rec + gl * RW;
        const int npat = rg[0];
        for (int kk = 0; kk < npat; ++kk, ++row) {
          const int32_t* pe = rg + 4 + DW + 5 * kk;
          const int len = T + pe[4];
          if (row % NWC == warp) {
            const int bmin = pe[3];
            const float* x0 = sd + (gl * kSubGroup + 0) * a.slot_w + (bmin - win[gl * kSubGroup + 0]);
            const float* x1 = sd + (gl * kSubGroup + 1) * a.slot_w + (bmin + pe[0] - win[gl * kSubGroup + 1]);
            const float* x2 = sd + (gl * kSubGroup + 2) * a.slot_w + (bmin + pe[1] - win[gl * kSubGroup + 2]);
            const float* x3 = sd + (gl * kSubGroup + 3) * a.slot_w + (bmin + pe[2] - win[gl * kSubGroup + 3]);
            double* pr = pbuf + poff;
            for (int tau = lane; tau < len; tau += 32) {
              double v = (double)x0[tau];
              v += (double)x1[tau];
              v += (double)x2[tau];
              v += (double)x3[tau];
              pr[tau] = v;
            }
          }
          poff += len;
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&pbar[0]);
    if (!mbar_wait(&pbar[0], k & 1, a.status)) { ok = false; break; }
    // stage 2: this warp's trial adds its pattern's row of each group at its shift
    if (dm < a.ndm) {
#pragma unroll
      for (int gl = 0; gl < NG; ++gl) {
        if (gl >= ng) break;
        const int32_t* rg = rec + gl * RW;
        const int e = rg[4 + dmw];
        const int pat = e >> 16, off = e & 0xffff;
        int rowoff = rowbase[gl];
        for (int kk = 0; kk < pat; ++kk) rowoff += T + rg[4 + DW + 5 * kk + 4];
        const double* pr = pbuf + rowoff + off + wbase;
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] += pr[32 * r];
      }
    }
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&pbar[1]);
      mbar_arrive(&empty[s]);
    }
    if (!mbar_wait(&pbar[1], k & 1, a.status)) { ok = false; break; }
  }
  if (!ok || dm >= a.ndm) return;
  float* out = static_cast<float*>(a.out) + (int64_t)dm * a.out_stride + a.out_start;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t t = t0 + wbase + 32 * r;
    if (t < a.nvalid) out[t] = (float)acc[r];
  }
}

}  // namespace spp
