// Host side of the persistent work-list DM-time kernel (k_dmt_wl) and the
// exposed corner turn / planar layout used to build batched work.
#include <algorithm>
#include <vector>

#include "spp_common.cuh"
#include "spp_dmt.cuh"

namespace spp {

struct WlVariant {
  int nb, acc, R, DW, TW, SLAB, STAGES;
  void (*fn)(const WlArgs);
  int planes;  // 1: bit-sliced over bit-plane rows (R = words per thread)
  int slot;    // > 0: kernel compiled for exactly this slot width (words)
};

template <int NB, int R, int DW, int TW, int SLAB, int STAGES, int ACC>
static WlVariant mkwl() {
  return WlVariant{NB, ACC, R, DW, TW, SLAB, STAGES, &k_dmt_wl<NB, R, DW, TW, SLAB, STAGES, ACC>, 0,
                   0};
}

template <int NB, int P, int DW, int TW, int STAGES, int SLAB, int SLOT = 0, int MINB = 0>
static WlVariant mkwlb() {
  constexpr int L = BitsLevels<NB>::kLevels;
  void (*fn)(const WlArgs) = &k_dmt_bits_wl<NB, P, DW, TW, STAGES, L, SLAB, SLOT>;
  if constexpr (MINB > 0) fn = &k_dmt_bits_wl_minb<NB, P, DW, TW, STAGES, L, SLAB, SLOT, MINB>;
  return WlVariant{NB, 0, P, DW, TW, SLAB, STAGES, fn, 1, SLOT};
}

#define SPP_WL_INT(NB)                                                                  \
  mkwl<NB, 2, 8, 1, 64, 3, 0>(), mkwl<NB, 1, 8, 1, 64, 3, 0>(), mkwl<NB, 2, 4, 2, 64, 3, 0>(), \
      mkwl<NB, 1, 4, 2, 64, 3, 0>()

static const std::vector<WlVariant>& wl_variants() {
  static const std::vector<WlVariant> v = {
      // fixed slot widths first (4 CTAs per SM), then runtime widths
      mkwlb<1, 2, 8, 1, 2, 32, 80, 4>(), mkwlb<1, 2, 8, 1, 2, 32, 128, 4>(),
      mkwlb<1, 2, 8, 1, 2, 64>(), mkwlb<1, 2, 8, 1, 3, 32>(),
      mkwlb<2, 2, 8, 1, 2, 32, 80, 4>(), mkwlb<2, 2, 8, 1, 2, 32, 128, 4>(),
      mkwlb<2, 2, 8, 1, 2, 64>(), mkwlb<2, 2, 8, 1, 3, 32>(),
      // bit-sliced 4- and 8-bit ahead of the SIMD kernels (faster at every span)
      mkwlb<4, 2, 8, 1, 2, 16, 96, 3>(), mkwlb<4, 2, 8, 1, 2, 16, 128, 3>(),
      mkwlb<4, 2, 8, 1, 2, 16>(),
      mkwlb<8, 2, 8, 1, 2, 16, 96, 2>(), mkwlb<8, 2, 8, 1, 2, 16, 0, 2>(),
      mkwlb<8, 1, 8, 1, 2, 16>(),
      SPP_WL_INT(1), SPP_WL_INT(2), SPP_WL_INT(4), SPP_WL_INT(8), SPP_WL_INT(16),
      mkwl<32, 8, 8, 1, 32, 2, SPP_ACC_KAHAN32>(), mkwl<32, 4, 8, 2, 32, 2, SPP_ACC_KAHAN32>(),
      mkwl<32, 8, 8, 1, 32, 2, SPP_ACC_F64>(),     mkwl<32, 4, 8, 2, 32, 2, SPP_ACC_F64>(),
  };
  return v;
}

static const WlVariant* wl_find(int nbits, int acc, int variant) {
  int k = 0;
  for (const auto& v : wl_variants()) {
    if (v.nb != nbits || (nbits == 32 && v.acc != acc)) continue;
    if (k == variant) return &v;
    ++k;
  }
  return nullptr;
}

static int spw_of_nb(int nb) { return nb == 32 ? 1 : 32 / nb; }
static int spw_wl(const WlVariant& v) { return v.planes ? 32 : spw_of_nb(v.nb); }

static int64_t wl_T(const WlVariant& v) { return (int64_t)v.TW * 32 * v.R * spw_wl(v); }

static int32_t wl_slot(const WlVariant& v, int32_t span) {
  const int spw = spw_wl(v);
  const int64_t w = wl_T(v) / spw + ceil_div(std::max<int32_t>(span, 0), spw) + 6 + v.R;
  const int32_t need = (int32_t)round_up(w, 4);
  if (v.slot > 0) return need <= v.slot ? v.slot : -1;  // fixed-width kernels
  return need;
}

static int64_t wl_smem(const WlVariant& v, int32_t slot_w) {
  const int64_t stage = v.planes ? bits_stage_bytes(v.nb, v.SLAB, slot_w, v.DW)
                                 : dmt_stage_bytes(v.SLAB, slot_w, v.DW);
  return (int64_t)v.STAGES * stage + 16 * v.STAGES + 8 + 2 * v.STAGES * 8;
}

static inline cudaStream_t stq(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace spp

using namespace spp;

extern "C" {

int spp_wl_num_variants(int nbits, int acc) {
  int n = 0;
  for (const auto& v : wl_variants())
    if (v.nb == nbits && (nbits != 32 || v.acc == acc)) ++n;
  return n;
}

int spp_wl_describe(int nbits, int acc, int variant, int32_t* cfg) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v || !cfg) return fail(SPP_ERR_ARG, "no work-list variant %d for nbits=%d acc=%d", variant, nbits, acc);
  cfg[0] = v->R; cfg[1] = v->DW; cfg[2] = v->TW; cfg[3] = v->SLAB; cfg[4] = v->STAGES;
  cfg[5] = (int32_t)wl_T(*v);
  cfg[6] = (v->DW * v->TW + 1) * 32;
  cfg[7] = spw_wl(*v) | (v->planes << 8);
  return SPP_OK;
}

int32_t spp_wl_slot_words(int nbits, int acc, int variant, int32_t span) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v) return -1;
  return wl_slot(*v, span);
}

int64_t spp_wl_smem_bytes(int nbits, int acc, int variant, int32_t slot_w) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v) return -1;
  return wl_smem(*v, slot_w);
}

int spp_wl_launch(int nbits, int acc, int variant, const void* items, int32_t nitems,
                  int32_t slot_w, int32_t* counter, uint32_t* status, int32_t nctas,
                  void* stream) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v) return fail(SPP_ERR_ARG, "no work-list variant %d for nbits=%d acc=%d", variant, nbits, acc);
  if (!items || !counter || nitems < 0 || slot_w <= 0 || (slot_w & 3))
    return fail(SPP_ERR_ARG, "bad work-list arguments");
  if (v->slot > 0 && slot_w != v->slot)
    return fail(SPP_ERR_ARG, "work-list variant %d takes slot width %d (got %d)", variant, v->slot,
                slot_w);
  if (nitems == 0) return SPP_OK;
  const int64_t smem = wl_smem(*v, slot_w);
  if (smem > 227 * 1024) return fail(SPP_ERR_UNSUPPORTED, "work list needs %lld B shared memory", (long long)smem);
  cudaStream_t st = stq(stream);
  int rc = SPP_OK;
  if (smem > 48 * 1024) {
    rc = set_smem_attr(reinterpret_cast<const void*>(v->fn), smem);
    if (rc) return rc;
  }
  const int threads = (v->DW * v->TW + 1) * 32;
  if (nctas <= 0) {
    int dev = 0, sms = 0, per = 0;
    rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
    if (rc) return rc;
    rc = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "sm count");
    if (rc) return rc;
    rc = cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, v->fn, threads, smem), "occupancy");
    if (rc) return rc;
    nctas = std::max(1, sms * std::max(per, 1));
  }
  nctas = std::min<int32_t>(nctas, nitems);
  rc = cuda_status(cudaMemsetAsync(counter, 0, sizeof(int32_t), st), "counter reset");
  if (rc) return rc;
  WlArgs w{};
  w.items = static_cast<const DmtItem*>(items);
  w.nitems = nitems;
  w.slot_w = slot_w;
  w.counter = counter;
  w.status = status;
  v->fn<<<nctas, threads, smem, st>>>(w);
  return cuda_status(cudaGetLastError(), "work-list launch");
}

int spp_planar_layout(int nbits, int64_t tile_T, int64_t nvalid, int32_t omin, int32_t omax,
                      int32_t slot_w, int64_t* halo, int64_t* pitch_w) {
  if (!halo || !pitch_w || tile_T <= 0 || slot_w <= 0) return fail(SPP_ERR_ARG, "bad layout arguments");
  if (nbits != 1 && nbits != 2 && nbits != 4 && nbits != 8 && nbits != 16 && nbits != 32)
    return fail(SPP_ERR_ARG, "bad nbits %d", nbits);
  const int spw = spw_of_nb(nbits);
  *halo = round_up(std::max<int64_t>(0, -(int64_t)omin), 4 * spw);
  const int64_t ntiles = ceil_div(std::max<int64_t>(nvalid, 1), tile_T);
  const int64_t last = ntiles * tile_T + std::max<int64_t>(0, omax) + *halo;
  *pitch_w = round_up(ceil_div(last, spw) + slot_w + 8, 4);
  return SPP_OK;
}

int spp_corner_turn(const void* in, int nbits, int bitorder, int64_t nchans, int64_t nsamps,
                    int64_t halo, void* planar, int64_t pitch_w, void* stream) {
  if (!in || !planar) return fail(SPP_ERR_ARG, "null pointer");
  if (nbits != 1 && nbits != 2 && nbits != 4 && nbits != 8 && nbits != 32)
    return fail(SPP_ERR_ARG, "bad nbits %d", nbits);
  if (nchans <= 0 || nsamps <= 0 || pitch_w <= 0 || (pitch_w & 3) || halo < 0)
    return fail(SPP_ERR_ARG, "bad shape");
  if (nbits < 8 && (nchans * nbits) % 8) return fail(SPP_ERR_ARG, "nchans*nbits must be a multiple of 8");
  cudaStream_t st = stq(stream);
  if (nbits == 32) {
    dim3 grid((unsigned)ceil_div(nchans, 32), (unsigned)std::min<int64_t>(ceil_div(pitch_w, 32), 65535));
    k_corner_turn_f32<<<grid, 256, 0, st>>>(static_cast<const float*>(in), nchans, nsamps, halo,
                                            static_cast<float*>(planar), pitch_w, nullptr, nullptr,
                                            nullptr);
  } else {
    dim3 grid((unsigned)ceil_div(nchans, kCtChans),
              (unsigned)std::min<int64_t>(ceil_div(pitch_w, kCtWords), 65535));
    const uint8_t* raw = static_cast<const uint8_t*>(in);
    uint32_t* pl = static_cast<uint32_t*>(planar);
    switch (nbits) {
      case 1: k_corner_turn_int<1><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w); break;
      case 2: k_corner_turn_int<2><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w); break;
      case 4: k_corner_turn_int<4><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w); break;
      default: k_corner_turn_int<8><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w); break;
    }
  }
  return cuda_status(cudaGetLastError(), "corner turn launch");
}

}  // extern "C"

extern "C" int32_t spp_wl_default_ctas(int nbits, int acc, int variant, int32_t slot_w) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v) return -1;
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  const int64_t smem = wl_smem(*v, slot_w);
  if (smem > 48 * 1024 && set_smem_attr(reinterpret_cast<const void*>(v->fn), smem)) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, v->fn, (v->DW * v->TW + 1) * 32, smem) !=
      cudaSuccess)
    return -1;
  return std::max(1, sms * std::max(per, 1));
}

extern "C" {

int spp_wl_planar_layout(int nbits, int acc, int variant, int64_t nvalid, int32_t omin,
                         int32_t omax, int32_t slot_w, int64_t* halo, int64_t* pitch_w,
                         int64_t* rows_per_chan) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v || !halo || !pitch_w || !rows_per_chan || slot_w <= 0) return fail(SPP_ERR_ARG, "bad layout arguments");
  const int spw = spw_wl(*v);
  const int64_t T = wl_T(*v);
  *halo = round_up(std::max<int64_t>(0, -(int64_t)omin), 4 * spw);
  const int64_t ntiles = ceil_div(std::max<int64_t>(nvalid, 1), T);
  const int64_t last = ntiles * T + std::max<int64_t>(0, omax) + *halo;
  *pitch_w = round_up(ceil_div(last, spw) + slot_w + 8, 4);
  *rows_per_chan = v->planes ? v->nb : 1;
  return SPP_OK;
}

int spp_wl_corner_turn(int nbits, int acc, int variant, const void* in, int bitorder,
                       int64_t nchans, int64_t nsamps, int64_t halo, void* planar,
                       int64_t pitch_w, void* stream) {
  const WlVariant* v = wl_find(nbits, acc, variant);
  if (!v) return fail(SPP_ERR_ARG, "no work-list variant %d for nbits=%d", variant, nbits);
  if (!v->planes) return spp_corner_turn(in, nbits, bitorder, nchans, nsamps, halo, planar, pitch_w, stream);
  if (!in || !planar || nchans <= 0 || nsamps <= 0 || (pitch_w & 3) || halo < 0 || (nchans * nbits) % 8)
    return fail(SPP_ERR_ARG, "bad corner-turn arguments");
  dim3 grid((unsigned)ceil_div(nchans, planes_ct_chans(nbits)),
            (unsigned)std::min<int64_t>(ceil_div(pitch_w, kPlaneWords), 65535));
  const uint8_t* raw = static_cast<const uint8_t*>(in);
  uint32_t* pl = static_cast<uint32_t*>(planar);
  cudaStream_t st = stq(stream);
  if (nbits == 1)
    k_corner_turn_planes<1><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w);
  else if (nbits == 2)
    k_corner_turn_planes<2><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w);
  else if (nbits == 4)
    k_corner_turn_planes<4><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w);
  else
    k_corner_turn_planes<8><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, halo, pl, pitch_w);
  return cuda_status(cudaGetLastError(), "plane corner turn launch");
}

}  // extern "C"
