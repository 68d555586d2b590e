// libsppgpu core: error state, unpack (R4), single-DM dedispersion (R2) and
// the DM-trial batch plan (R3).  Host code for the kernels in spp_dmt.cuh.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "spp_common.cuh"
#include "spp_dmt.cuh"

namespace spp {

int launch_single8(const uint8_t* raw, int64_t nchans, int64_t nsamps, const int32_t* delays,
                   int32_t dlo, int32_t dhi, float* out, int64_t out_start, int64_t nvalid,
                   uint32_t* status, cudaStream_t st);
int launch_single8_hd(const uint8_t* raw, int64_t nchans, int64_t nsamps, const int32_t* delays_host,
                      float* out, int64_t out_start, int64_t nvalid, cudaStream_t st);

static thread_local char g_err[1024] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SPP_OK;
  return fail(SPP_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Raises a kernel's dynamic shared memory limit once per (device, kernel):
// later calls with a size at or below the recorded one issue no CUDA call, so
// launches stay legal inside CUDA-graph capture after one eager run.
int set_smem_attr(const void* fn, int64_t bytes) {
  static std::mutex mu;
  static std::vector<std::tuple<int, const void*, int64_t>> done;
  int dev = 0;
  int rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(mu);
  for (auto& e : done)
    if (std::get<0>(e) == dev && std::get<1>(e) == fn && std::get<2>(e) >= bytes) return SPP_OK;
  rc = cuda_status(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
                   "cudaFuncSetAttribute");
  if (rc) return rc;
  done.emplace_back(dev, fn, bytes);
  return SPP_OK;
}

static inline bool valid_nbits(int nbits) {
  return nbits == 1 || nbits == 2 || nbits == 4 || nbits == 8 || nbits == 32;
}

// ---------------------------------------------------------------------------
// R4: standalone unpack (kernels.unpack{1,2,4}_8_{big,little})
// ---------------------------------------------------------------------------
template <int NB>
__global__ void k_unpack(const uint8_t* __restrict__ in, int64_t nbytes, int bitorder,
                         uint8_t* __restrict__ out) {
  constexpr int per = 8 / NB;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nbytes;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t b = in[i];
#pragma unroll
    for (int k = 0; k < per; ++k) out[i * per + k] = (uint8_t)field_of<NB>(b, k, bitorder);
  }
}

// ---------------------------------------------------------------------------
// DMT kernel variants
// ---------------------------------------------------------------------------
struct Variant {
  int nb, acc, R, DW, TW, SLAB, STAGES;
  void (*fn)(const DmtArgs);
  int single;  // 1: meant for one DM (time-split warps)
  int planes;  // 1: bit-sliced kernel over bit-plane rows (R = words per thread)
  int slot;    // > 0: kernel compiled for exactly this slot width (words)
  int pairs = 0;  // 1: 2-bit channel-pair kernel over pair-sum rows (three planes)
};

template <int NB, int R, int DW, int TW, int SLAB, int STAGES, int ACC>
static Variant mk(int single) {
  return Variant{NB, ACC, R, DW, TW, SLAB, STAGES, &k_dmt<NB, R, DW, TW, SLAB, STAGES, ACC>,
                 single, 0, 0};
}

// Bit-sliced counters hold sums below 2^bit_levels(nbits).
static int bit_levels(int nbits) {
  return nbits == 8 ? BitsLevels<8>::kLevels : nbits == 4 ? BitsLevels<4>::kLevels : BitsLevels<2>::kLevels;
}

template <int NB, int P, int DW, int TW, int STAGES, int SLAB = 64, int SLOT = 0, int MINB = 0>
static Variant mkb() {
  constexpr int L = BitsLevels<NB>::kLevels;
  void (*fn)(const DmtArgs) = &k_dmt_bits<NB, P, DW, TW, STAGES, L, SLAB, SLOT>;
  if constexpr (MINB > 0) fn = &k_dmt_bits_minb<NB, P, DW, TW, STAGES, L, SLAB, SLOT, MINB>;
  return Variant{NB, 0, P, DW, TW, SLAB, STAGES, fn, 0, 1, SLOT};
}

// Channel-pair kernels (2-bit data): SLAB pairs per slab, two staged rows
// per pair.
template <int P, int DW, int TW, int STAGES, int SLAB, int SLOT = 0, int MINB = 0>
static Variant mkp() {
  constexpr int L = BitsLevels<3>::kLevels;
  void (*fn)(const DmtArgs) = &k_dmt_pairs<P, DW, TW, STAGES, L, SLAB, SLOT>;
  if constexpr (MINB > 0) fn = &k_dmt_pairs_minb<P, DW, TW, STAGES, L, SLAB, SLOT, MINB>;
  Variant v{2, 0, P, DW, TW, SLAB, STAGES, fn, 0, 1, SLOT};
  v.pairs = 1;
  return v;
}

#define SPP_INT_VARIANTS(NB)                    \
  mk<NB, 2, 8, 1, 64, 3, 0>(0), mk<NB, 1, 8, 1, 64, 3, 0>(0), mk<NB, 2, 4, 2, 64, 3, 0>(0), \
      mk<NB, 1, 16, 1, 64, 3, 0>(0), mk<NB, 2, 1, 4, 64, 3, 0>(1), mk<NB, 1, 1, 4, 64, 3, 0>(1)

static const std::vector<Variant>& variants() {
  static const std::vector<Variant> v = {
      // bit-sliced (1- and 2-bit data)
      // fixed slot widths first: 32-channel slabs keep 3-4 CTAs resident per SM
      mkb<2, 2, 8, 1, 2, 32, 80, 4>(), mkb<2, 2, 8, 1, 2, 32, 80>(), mkb<2, 2, 8, 1, 3, 32, 80>(),
      mkb<2, 2, 8, 1, 2, 32, 96>(), mkb<2, 2, 8, 1, 2, 32, 128>(),
      mkb<2, 2, 8, 1, 2, 64, 80>(), mkb<2, 2, 8, 1, 2, 64, 96>(),
      mkb<2, 3, 8, 1, 2, 32, 112, 3>(), mkb<2, 3, 8, 1, 2, 32, 112, 2>(),
      mkb<2, 2, 8, 1, 2>(), mkb<2, 2, 8, 1, 3, 32>(), mkb<2, 2, 8, 1, 2, 32>(),
      mkb<2, 4, 8, 1, 2, 32>(), mkb<2, 2, 16, 1, 2, 32>(), mkb<2, 1, 8, 1, 3>(),
      // channel pairs summed once per relative delay (2-bit DM grids whose
      // adjacent channels differ by few distinct delays)
      mkp<3, 8, 1, 2, 8, 112, 3>(), mkp<3, 8, 1, 3, 8, 112, 3>(), mkp<3, 8, 1, 2, 16, 112, 2>(),
      mkp<2, 8, 1, 2, 16, 80, 3>(), mkp<3, 8, 1, 2, 16>(), mkp<2, 8, 1, 3, 8>(),
      mkb<1, 2, 8, 1, 2, 32, 80>(), mkb<1, 2, 8, 1, 2, 32, 128>(),
      mkb<1, 2, 8, 1, 2>(), mkb<1, 2, 8, 1, 3, 32>(), mkb<1, 4, 8, 1, 2, 32>(),
      SPP_INT_VARIANTS(1),
      SPP_INT_VARIANTS(2),
      // bit-sliced 4-bit (four plane rows per channel; 16-channel slabs keep
      // a stage's planes within a third of shared memory): 1.8-2.3x the SIMD
      // kernels' adds/s, so they come first for 4-bit data
      mkb<4, 2, 8, 1, 2, 16, 96, 3>(), mkb<4, 2, 8, 1, 2, 16>(), mkb<4, 3, 8, 1, 2, 16, 112, 2>(),
      mkb<4, 2, 8, 1, 2, 32>(), mkb<4, 1, 8, 1, 3, 16>(),
      SPP_INT_VARIANTS(4),
      // bit-sliced 8-bit (eight plane rows per channel, 20-level counters):
      // 1.6-2.8x the SIMD byte-lane kernels, so they come first for 8-bit data
      mkb<8, 2, 8, 1, 2, 16, 96, 2>(), mkb<8, 2, 8, 1, 2, 16, 0, 2>(), mkb<8, 1, 8, 1, 2, 16>(),
      mkb<8, 1, 8, 1, 3, 16>(),
      SPP_INT_VARIANTS(8),
      mk<8, 4, 1, 4, 16, 3, 0>(1),
      // float32 input, compensated fp32
      mk<32, 8, 8, 1, 32, 2, SPP_ACC_KAHAN32>(0),
      mk<32, 4, 8, 2, 32, 2, SPP_ACC_KAHAN32>(0),
      mk<32, 8, 16, 1, 32, 2, SPP_ACC_KAHAN32>(0),
      mk<32, 8, 4, 1, 16, 2, SPP_ACC_KAHAN32>(0),
      mk<32, 4, 1, 4, 32, 2, SPP_ACC_KAHAN32>(1),
      mk<32, 2, 1, 4, 32, 2, SPP_ACC_KAHAN32>(1),
      mk<32, 16, 4, 1, 16, 2, SPP_ACC_KAHAN32>(0),
      mk<32, 8, 2, 1, 16, 2, SPP_ACC_KAHAN32>(0),
      mk<32, 16, 2, 1, 16, 2, SPP_ACC_KAHAN32>(0),
      // float32 input, fp64 accumulator (channel-ordered sums: the reference's)
      mk<32, 16, 4, 1, 16, 2, SPP_ACC_F64>(0),
      mk<32, 16, 2, 1, 16, 2, SPP_ACC_F64>(0),
      mk<32, 8, 2, 1, 16, 2, SPP_ACC_F64>(0),
      mk<32, 8, 8, 1, 32, 2, SPP_ACC_F64>(0),
      mk<32, 4, 8, 2, 32, 2, SPP_ACC_F64>(0),
      mk<32, 8, 4, 1, 16, 2, SPP_ACC_F64>(0),
      mk<32, 4, 1, 4, 32, 2, SPP_ACC_F64>(1),
      mk<32, 2, 1, 4, 32, 2, SPP_ACC_F64>(1),
  };
  return v;
}

static inline int spw_of(int nb) { return nb == 32 ? 1 : 32 / nb; }
static inline int spw_v(const Variant& v) { return v.planes ? 32 : spw_of(v.nb); }
static inline int64_t tile_T(const Variant& v) {
  return (int64_t)v.TW * 32 * v.R * spw_v(v);
}

static int slot_words(const Variant& v, int32_t span) {
  const int spw = spw_v(v);
  const int64_t w = tile_T(v) / spw + ceil_div(std::max<int32_t>(span, 0), spw) + 6 + v.R;
  const int need = (int)round_up(w, 4);
  if (v.slot > 0) return need <= v.slot ? v.slot : -1;  // fixed-width kernels
  return need;
}

static int64_t smem_bytes(const Variant& v, int slot_w) {
  if (v.pairs)
    return v.STAGES * pair_stage_bytes(v.SLAB, slot_w, v.DW) + 8 + 2 * v.STAGES * 8 +
           pair_hi_bytes(v.R, v.DW * v.TW);
  if (v.planes) return v.STAGES * bits_stage_bytes(v.nb, v.SLAB, slot_w, v.DW) + 8 + 2 * v.STAGES * 8;
  return v.STAGES * dmt_stage_bytes(v.SLAB, slot_w, v.DW) + 8 + 2 * v.STAGES * 8;
}

static constexpr int64_t kMaxSmem = 227 * 1024;

// Planar geometry for one execution.
struct Geometry {
  int planes;
  int spw;
  int64_t halo;     // samples
  int64_t pitch_w;  // words per channel row
  int64_t bytes;    // nchans * pitch_w * 4
  int64_t ntiles_t;
  int64_t nvalid;
};

// omin/omax: range of the signed offsets applied to t (sign * delay).
static Geometry geometry(const Variant& v, int64_t nchans, int64_t nsamps, int64_t nvalid,
                         int32_t omin, int32_t omax, int slot_w) {
  Geometry g{};
  g.planes = v.planes;
  g.spw = spw_v(v);
  g.nvalid = nvalid;
  g.halo = round_up(std::max<int64_t>(0, -(int64_t)omin), 4 * g.spw);
  g.ntiles_t = ceil_div(std::max<int64_t>(nvalid, 1), tile_T(v));
  const int64_t last = g.ntiles_t * tile_T(v) + std::max<int64_t>(0, omax) + g.halo;
  g.pitch_w = round_up(ceil_div(last, g.spw) + slot_w + 8, 4);
  g.bytes = nchans * (v.planes ? v.nb : 1) * g.pitch_w * 4;
  (void)nsamps;
  return g;
}

static int ensure_smem(const Variant& v, int64_t bytes) {
  if (bytes > kMaxSmem)
    return fail(SPP_ERR_UNSUPPORTED, "DM tile needs %lld B of shared memory (> %lld)",
                (long long)bytes, (long long)kMaxSmem);
  if (bytes > 48 * 1024) return set_smem_attr(reinterpret_cast<const void*>(v.fn), bytes);
  return SPP_OK;
}

static int launch_corner_turn(int nb, const void* in, int bitorder, int64_t nchans,
                              int64_t nsamps, const Geometry& g, void* planar, cudaStream_t st,
                              const double* zdm = nullptr, const float* chanwts = nullptr,
                              const float* bpass = nullptr, uint32_t* special = nullptr) {
  if (g.planes) {
    dim3 grid((unsigned)ceil_div(nchans, planes_ct_chans(nb)),
              (unsigned)std::min<int64_t>(ceil_div(g.pitch_w, kPlaneWords), 65535));
    const uint8_t* raw = static_cast<const uint8_t*>(in);
    uint32_t* pl = static_cast<uint32_t*>(planar);
    if (nb == 1)
      k_corner_turn_planes<1><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w);
    else if (nb == 2)
      k_corner_turn_planes<2><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w);
    else if (nb == 4)
      k_corner_turn_planes<4><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w);
    else if (nb == 8)
      k_corner_turn_planes<8><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w);
    else
      return fail(SPP_ERR_UNSUPPORTED, "bit planes for nbits=%d", nb);
  } else if (nb == 32) {
    dim3 grid((unsigned)ceil_div(nchans, 32),
              (unsigned)std::min<int64_t>(ceil_div(g.pitch_w, 32), 65535));
    k_corner_turn_f32<<<grid, 256, 0, st>>>(static_cast<const float*>(in), nchans, nsamps,
                                            g.halo, static_cast<float*>(planar), g.pitch_w,
                                            zdm, chanwts, bpass, special);
  } else {
    dim3 grid((unsigned)ceil_div(nchans, kCtChans),
              (unsigned)std::min<int64_t>(ceil_div(g.pitch_w, kCtWords), 65535));
    const uint8_t* raw = static_cast<const uint8_t*>(in);
    uint32_t* pl = static_cast<uint32_t*>(planar);
    switch (nb) {
      case 1: k_corner_turn_int<1><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w); break;
      case 2: k_corner_turn_int<2><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w); break;
      case 4: k_corner_turn_int<4><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w); break;
      default: k_corner_turn_int<8><<<grid, 256, 0, st>>>(raw, nchans, nsamps, bitorder, g.halo, pl, g.pitch_w); break;
    }
  }
  return cuda_status(cudaGetLastError(), "corner turn launch");
}

static int launch_dmt(const Variant& v, const DmtArgs& a, int64_t ntiles_t, int64_t ndm,
                      cudaStream_t st) {
  const int64_t smem = smem_bytes(v, a.slot_w);
  int rc = ensure_smem(v, smem);
  if (rc) return rc;
  dim3 grid((unsigned)ceil_div(ndm, v.DW), (unsigned)ntiles_t);
  if (ntiles_t > 65535)
    return fail(SPP_ERR_UNSUPPORTED, "too many time tiles (%lld)", (long long)ntiles_t);
  const int threads = (v.DW * v.TW + 1) * 32;
  v.fn<<<grid, threads, smem, st>>>(a);
  return cuda_status(cudaGetLastError(), "dmt launch");
}

// Single-DM shape: the largest time tile that still yields >= 2 CTAs per SM
// (148 SMs), else the smallest tile.  Shapes are the same for both float
// accumulators, so the workspace size does not depend on `acc`.
static int pick_single_variant(int nb, int acc, int64_t nvalid) {
  const auto& vs = variants();
  int best_big = -1, best_small = -1;
  for (int i = 0; i < (int)vs.size(); ++i) {
    const Variant& v = vs[i];
    if (!v.single || v.nb != nb || (nb == 32 && v.acc != acc)) continue;
    if (smem_bytes(v, slot_words(v, 0)) > kMaxSmem) continue;
    const int64_t T = tile_T(v);
    if (ceil_div(nvalid, T) >= 296 && (best_big < 0 || T > tile_T(vs[best_big]))) best_big = i;
    if (best_small < 0 || T < tile_T(vs[best_small])) best_small = i;
  }
  return best_big >= 0 ? best_big : best_small;
}

}  // namespace spp

using namespace spp;

// ---------------------------------------------------------------------------
// extern "C" entry points
// ---------------------------------------------------------------------------
extern "C" {

const char* spp_last_error_string(void) { return g_err; }

int spp_version(void) { return 10000; }

int spp_status_read(const void* workspace, uint32_t* host_out, void* stream) {
  if (!workspace || !host_out) return fail(SPP_ERR_ARG, "spp_status_read: null pointer");
  cudaStream_t st = as_stream(stream);
  int rc = cuda_status(cudaMemcpyAsync(host_out, workspace, 16, cudaMemcpyDeviceToHost, st),
                       "status copy");
  if (rc) return rc;
  rc = cuda_status(cudaStreamSynchronize(st), "status sync");
  if (rc) return rc;
  if (host_out[0] != 0)
    return fail(SPP_ERR_DEVICE, "device status 0x%x (block %u, detail 0x%x)", host_out[0],
                host_out[1], host_out[2]);
  return SPP_OK;
}

int spp_status_clear(void* workspace, void* stream) {
  if (!workspace) return fail(SPP_ERR_ARG, "spp_status_clear: null pointer");
  return cuda_status(cudaMemsetAsync(workspace, 0, 16, as_stream(stream)), "status clear");
}

int spp_host_register(void* ptr, int64_t bytes) {
  if (!ptr || bytes <= 0) return fail(SPP_ERR_ARG, "spp_host_register: null pointer or size <= 0");
  const cudaError_t e = cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();  // a refused registration must not surface at the next launch check
    return fail(SPP_ERR_CUDA, "cudaHostRegister: %s", cudaGetErrorString(e));
  }
  return SPP_OK;
}

int spp_host_unregister(void* ptr) {
  if (!ptr) return fail(SPP_ERR_ARG, "spp_host_unregister: null pointer");
  const cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SPP_ERR_CUDA, "cudaHostUnregister: %s", cudaGetErrorString(e));
  }
  return SPP_OK;
}

int spp_unpack(const uint8_t* in, int64_t nbytes, int nbits, int bitorder, uint8_t* out,
               void* stream) {
  if (nbytes < 0) return fail(SPP_ERR_ARG, "nbytes < 0");
  if (nbytes == 0) return SPP_OK;
  if (!in || !out) return fail(SPP_ERR_ARG, "spp_unpack: null pointer");
  if (bitorder != SPP_BITORDER_BIG && bitorder != SPP_BITORDER_LITTLE)
    return fail(SPP_ERR_ARG, "bad bitorder %d", bitorder);
  cudaStream_t st = as_stream(stream);
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(nbytes, threads), 148 * 32);
  switch (nbits) {
    case 1: k_unpack<1><<<(unsigned)blocks, threads, 0, st>>>(in, nbytes, bitorder, out); break;
    case 2: k_unpack<2><<<(unsigned)blocks, threads, 0, st>>>(in, nbytes, bitorder, out); break;
    case 4: k_unpack<4><<<(unsigned)blocks, threads, 0, st>>>(in, nbytes, bitorder, out); break;
    default: return fail(SPP_ERR_ARG, "unpack: nbits must be 1, 2 or 4 (got %d)", nbits);
  }
  return cuda_status(cudaGetLastError(), "unpack launch");
}

// ---------------------------------------------------------------------------
// R2: single DM
// ---------------------------------------------------------------------------
static int single_setup(int nbits, int64_t nchans, int64_t nsamps, int32_t dmin, int32_t dmax,
                        int acc, const Variant** vout, Geometry* gout, int* slot_out) {
  if (!valid_nbits(nbits)) return fail(SPP_ERR_ARG, "nbits must be 1, 2, 4, 8 or 32 (got %d)", nbits);
  if (nchans <= 0 || nsamps < 0) return fail(SPP_ERR_ARG, "bad shape nchans=%lld nsamps=%lld", (long long)nchans, (long long)nsamps);
  if (nbits < 8 && (nchans * nbits) % 8 != 0)
    return fail(SPP_ERR_ARG, "nchans*nbits must be a multiple of 8");
  if (dmin > dmax) return fail(SPP_ERR_ARG, "delay_min > delay_max");
  if (nchans > INT32_MAX) return fail(SPP_ERR_ARG, "nchans too large");
  const int64_t maxabs = std::max<int64_t>(std::llabs(dmin), std::llabs(dmax));
  const int64_t nvalid = nsamps - maxabs;
  const int vi = pick_single_variant(nbits, acc, std::max<int64_t>(nvalid, 1));
  if (vi < 0) return fail(SPP_ERR_UNSUPPORTED, "no kernel for nbits=%d acc=%d", nbits, acc);
  const Variant& v = variants()[vi];
  const int slot = slot_words(v, 0);
  *vout = &v;
  *slot_out = slot;
  *gout = geometry(v, nchans, nsamps, nvalid, dmin, dmax, slot);
  return SPP_OK;
}

int64_t spp_dedisperse_workspace_bytes(int nbits, int64_t nchans, int64_t nsamps,
                                       int32_t delay_min, int32_t delay_max) {
  const Variant* v;
  Geometry g;
  int slot;
  if (single_setup(nbits, nchans, nsamps, delay_min, delay_max, SPP_ACC_F64, &v, &g, &slot))
    return -1;
  return kStatusBytes + g.bytes;
}

int spp_dedisperse(const void* in, int nbits, int bitorder, int64_t nchans, int64_t nsamps,
                   const int32_t* delays, int32_t delay_min, int32_t delay_max, float* out,
                   int64_t out_len, int64_t out_start, int acc, void* workspace,
                   int64_t workspace_bytes, void* stream) {
  if (!in || !delays || !out || !workspace) return fail(SPP_ERR_ARG, "spp_dedisperse: null pointer");
  if (acc != SPP_ACC_F64 && acc != SPP_ACC_KAHAN32) return fail(SPP_ERR_ARG, "bad acc %d", acc);
  const Variant* v;
  Geometry g;
  int slot;
  int rc = single_setup(nbits, nchans, nsamps, delay_min, delay_max, acc, &v, &g, &slot);
  if (rc) return rc;
  if (g.nvalid <= 0) return SPP_OK;  // reference: prange over a non-positive count
  if (-(int64_t)delay_min > nsamps)
    return fail(SPP_ERR_DELAY, "negative delay %d reaches before the block", delay_min);
  if (out_start < 0 || out_start + g.nvalid > out_len)
    return fail(SPP_ERR_SIZE, "output too small: out_start %lld + %lld samples > out_len %lld",
                (long long)out_start, (long long)g.nvalid, (long long)out_len);
  if (workspace_bytes < kStatusBytes + g.bytes)
    return fail(SPP_ERR_SIZE, "workspace %lld B < required %lld B", (long long)workspace_bytes,
                (long long)(kStatusBytes + g.bytes));
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return fail(SPP_ERR_ALIGN, "workspace must be 256-B aligned");
  cudaStream_t st = as_stream(stream);
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  if (nbits == 8) {
    // one pass over the raw block when the delay spread fits the staging buffer
    rc = launch_single8(static_cast<const uint8_t*>(in), nchans, nsamps, delays, delay_min,
                        delay_max, out, out_start, g.nvalid, reinterpret_cast<uint32_t*>(ws), st);
    if (rc != SPP_ERR_UNSUPPORTED) return rc;
  }
  void* planar = ws + kStatusBytes;
  rc = launch_corner_turn(nbits, in, bitorder, nchans, nsamps, g, planar, st);
  if (rc) return rc;
  DmtArgs a{};
  a.planar = planar;
  a.pitch_w = g.pitch_w;
  a.halo = g.halo;
  a.nchans = (int32_t)nchans;
  a.delays = delays;
  a.dpitch = nchans;
  a.ndm = 1;
  a.sign = 1;
  a.dlo = delay_min;
  a.dhi = delay_max;
  a.span_max = 0;
  a.slot_w = slot;
  a.out = out;
  a.out_kind = SPP_OUT_F32;
  a.out_stride = 0;
  a.out_start = out_start;
  a.nvalid = g.nvalid;
  a.status = reinterpret_cast<uint32_t*>(ws);
  return launch_dmt(*v, a, g.ntiles_t, 1, st);
}

int spp_dedisperse_hd(const void* in, int nbits, int64_t nchans, int64_t nsamps,
                      const int32_t* delays_host, float* out, int64_t out_len, int64_t out_start,
                      void* stream) {
  if (!in || !delays_host || !out) return fail(SPP_ERR_ARG, "spp_dedisperse_hd: null pointer");
  if (nbits != 8) return fail(SPP_ERR_UNSUPPORTED, "host-table path covers 8-bit data");
  if (nchans <= 0 || nsamps <= 0) return fail(SPP_ERR_ARG, "bad shape");
  const int32_t dmin = *std::min_element(delays_host, delays_host + nchans);
  const int32_t dmax = *std::max_element(delays_host, delays_host + nchans);
  const int64_t maxabs = std::max<int64_t>(std::llabs(dmin), std::llabs(dmax));
  const int64_t nvalid = nsamps - maxabs;
  if (nvalid <= 0) return SPP_OK;  // reference: prange over a non-positive count
  if (-(int64_t)dmin > nsamps)
    return fail(SPP_ERR_DELAY, "negative delay %d reaches before the block", dmin);
  if (out_start < 0 || out_start + nvalid > out_len)
    return fail(SPP_ERR_SIZE, "output too small: out_start %lld + %lld samples > out_len %lld",
                (long long)out_start, (long long)nvalid, (long long)out_len);
  const int rc = launch_single8_hd(static_cast<const uint8_t*>(in), nchans, nsamps, delays_host,
                                   out, out_start, nvalid, as_stream(stream));
  if (rc == SPP_ERR_UNSUPPORTED)
    return fail(rc, "host-table path needs nchans %% 32 == 0, nchans <= 1024, a 16-B aligned "
                "block and every slab resident in shared memory");
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Single-DM dedispersion without allocation.
//
// For callers that must not allocate device memory once they are running --
// e.g. a real-time search pipeline that reserves its device memory at
// start-up and treats any later cudaMalloc (which can synchronise the device
// and can fail under memory pressure) as an error, or a host framework whose
// own allocator owns the device memory and hands out only input and output
// buffers.  The scratch that spp_dedisperse takes as `workspace` lives here
// in a fixed device array instead.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocScratchBytes = 32ll << 20;  // 32 MiB per device
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device, looked up
// once per device (the symbol name is only a host-side handle).
int noalloc_scratch(void** out) {
  int dev = 0;
  int rc = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= kMaxDevices) return fail(SPP_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    rc = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress");
    if (rc) return rc;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return SPP_OK;
}

}  // namespace

extern "C" {

int64_t spp_dedisperse_noalloc_max_bytes(void) { return kNoAllocScratchBytes; }

int spp_dedisperse_noalloc(const void* in, int nbits, int bitorder, int64_t nchans,
                           int64_t nsamps, const int32_t* delays, int32_t delay_min,
                           int32_t delay_max, float* out, int64_t out_len, int64_t out_start,
                           int acc, void* stream) {
  if (!in || !delays || !out) return fail(SPP_ERR_ARG, "spp_dedisperse_noalloc: null pointer");
  if (acc != SPP_ACC_F64 && acc != SPP_ACC_KAHAN32) return fail(SPP_ERR_ARG, "bad acc %d", acc);
  const Variant* v;
  Geometry g;
  int slot;
  int rc = single_setup(nbits, nchans, nsamps, delay_min, delay_max, acc, &v, &g, &slot);
  if (rc) return rc;
  if (g.nvalid <= 0) return SPP_OK;
  if (out_start < 0 || out_start + g.nvalid > out_len)
    return fail(SPP_ERR_SIZE, "output too small: out_start %lld + %lld samples > out_len %lld",
                (long long)out_start, (long long)g.nvalid, (long long)out_len);
  const int64_t need = kStatusBytes + g.bytes;
  if (need > kNoAllocScratchBytes)
    return fail(SPP_ERR_SIZE,
                "block needs %lld B of scratch, above the fixed %lld B of the no-allocation "
                "entry point: use spp_dedisperse with a workspace, or smaller blocks",
                (long long)need, (long long)kNoAllocScratchBytes);
  void* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  uint8_t* ws = static_cast<uint8_t*>(base);
  // the status block must start at zero; the planar rows are fully rewritten
  rc = cuda_status(cudaMemsetAsync(ws, 0, kStatusBytes, st), "status clear");
  if (rc) return rc;
  void* planar = ws + kStatusBytes;
  rc = launch_corner_turn(nbits, in, bitorder, nchans, nsamps, g, planar, st);
  if (rc) return rc;
  DmtArgs a{};
  a.planar = planar;
  a.pitch_w = g.pitch_w;
  a.halo = g.halo;
  a.nchans = (int32_t)nchans;
  a.delays = delays;
  a.dpitch = nchans;
  a.ndm = 1;
  a.sign = 1;
  a.dlo = delay_min;
  a.dhi = delay_max;
  a.span_max = 0;
  a.slot_w = slot;
  a.out = out;
  a.out_kind = SPP_OUT_F32;
  a.out_stride = 0;
  a.out_start = out_start;
  a.nvalid = g.nvalid;
  a.status = reinterpret_cast<uint32_t*>(ws);
  return launch_dmt(*v, a, g.ntiles_t, 1, st);
}

// The status words of the last spp_dedisperse_noalloc call on the current
// device sit at the head of the fixed array, where the caller has no pointer
// to them; this copies them out (synchronising `stream`).
int spp_dedisperse_noalloc_status_read(uint32_t* host_out, void* stream) {
  if (!host_out) return fail(SPP_ERR_ARG, "spp_dedisperse_noalloc_status_read: null pointer");
  void* base = nullptr;
  const int rc = noalloc_scratch(&base);
  if (rc) return rc;
  return spp_status_read(base, host_out, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// R3: DM-trial batch plan
// ---------------------------------------------------------------------------
struct spp_dmt_plan {
  int nbits, bitorder, mode, out_kind, acc;
  int64_t nchans, nsamps_max, ndm;
  int32_t* d_delays = nullptr;  // device, ndm x dpitch (raw delays)
  int64_t dpitch;
  int32_t dmin, dmax;  // raw delay range
  int32_t omin, omax;  // range of sign * delay
  int32_t maxabs;
  std::vector<int> cands;      // candidate variant indices
  std::vector<int32_t> spans;  // span per candidate
  int cur = 0;                 // index into cands
  // channel pairs (2-bit): rows (pair k, relative offset r) and each DM's row
  // per pair; empty when the table has too many distinct offsets
  int64_t nprows = 0;
  int2* d_pair_src = nullptr;      // device, nprows x (k, r)
  std::vector<int32_t> pair_rows;  // host, ndm x nchans/2
  std::vector<int32_t> delays_h;   // host copy of the table while pair kernels are offered
  // per candidate (nullptr until a pair kernel is first selected): staging tables
  std::vector<int2*> pair_off, pair_ent;
  // optional per-kernel timing: events (start, after corner turn, end) per execute
  bool timing = false;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
};

static cudaEvent_t plan_event(spp_dmt_plan* p) {
  if (p->evused == p->evpool.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    p->evpool.push_back(e);
  }
  return p->evpool[p->evused++];
}

static int plan_sign(const spp_dmt_plan* p) { return p->mode == SPP_MODE_ROLL ? -1 : 1; }

static int64_t plan_nvalid(const spp_dmt_plan* p, int64_t nsamps) {
  return p->mode == SPP_MODE_ROLL ? nsamps : nsamps - p->maxabs;
}

// Staging tables of a pair kernel with DW trials per tile, SLAB pairs per
// slab and slot_w words per staged row.  Per (tile, slab): the DW x SLAB
// decoded offsets (staged row x 3 x slot_w + word, bit shift) and the
// 2 x SLAB staged rows (pair-sum row, window start word relative to the time
// tile; -1: unused).  The window of pair k starts at the 4-word boundary at
// or below the tile's smallest offset of channel 2k; tiles are multiples of
// 128 samples, so the same tables serve every time tile.
static int pair_tables(spp_dmt_plan* p, const int32_t* delays_host, int dw, int slab, int slot_w,
                       int2** d_off, int2** d_ent) {
  const int64_t np = p->nchans / 2, ndm = p->ndm;
  const int64_t ntile = ceil_div(ndm, dw), nslab = ceil_div(np, slab);
  const int sign = plan_sign(p);
  const int64_t halo = round_up(std::max<int64_t>(0, -(int64_t)p->omin), 128);
  std::vector<int2> off((size_t)(ntile * nslab * dw * slab), make_int2(0, 0));
  std::vector<int2> ent((size_t)(ntile * nslab * 2 * slab), make_int2(-1, 0));
  for (int64_t t = 0; t < ntile; ++t) {
    for (int64_t k = 0; k < nslab; ++k) {
      const int64_t blk = t * nslab + k;
      int e = 0;
      for (int64_t j = 0; j < slab && k * slab + j < np; ++j) {
        const int64_t pr = k * slab + j;
        int32_t dv[64], rv[64], u[3];
        int nu = 0;
        int32_t mn = INT32_MAX;
        for (int i = 0; i < dw; ++i) {
          const int64_t dm = std::min<int64_t>(t * dw + i, ndm - 1);
          dv[i] = sign * delays_host[dm * p->nchans + 2 * pr];
          rv[i] = p->pair_rows[dm * np + pr];
          mn = std::min(mn, dv[i]);
          bool seen = false;
          for (int m = 0; m < nu; ++m) seen = seen || u[m] == rv[i];
          if (!seen) {
            if (nu == 3) return fail(SPP_ERR_UNSUPPORTED, "pair %lld: more than 3 rows in a tile", (long long)pr);
            u[nu++] = rv[i];
          }
        }
        if (e + nu > 2 * slab) return fail(SPP_ERR_UNSUPPORTED, "pair slab needs more than %d rows", 2 * slab);
        std::sort(u, u + nu);
        const int64_t wsrel = ((mn + halo) / 32) & ~int64_t(3);  // mn + halo >= 0
        const int64_t base = wsrel * 32 - halo;
        for (int m = 0; m < nu; ++m) ent[blk * 2 * slab + e + m] = make_int2(u[m], (int)wsrel);
        for (int i = 0; i < dw; ++i) {
          int m = 0;
          while (u[m] != rv[i]) ++m;
          const int64_t o = dv[i] - base;
          off[(blk * dw + i) * slab + j] =
              make_int2((int)((e + m) * 3 * slot_w + (o >> 5)), (int)(o & 31));
        }
        e += nu;
      }
    }
  }
  cudaError_t err = cudaMalloc(d_off, sizeof(int2) * off.size());
  if (err == cudaSuccess) err = cudaMalloc(d_ent, sizeof(int2) * ent.size());
  if (err == cudaSuccess)
    err = cudaMemcpy(*d_off, off.data(), sizeof(int2) * off.size(), cudaMemcpyHostToDevice);
  if (err == cudaSuccess)
    err = cudaMemcpy(*d_ent, ent.data(), sizeof(int2) * ent.size(), cudaMemcpyHostToDevice);
  if (err != cudaSuccess) {  // leave both unset so a later selection retries
    if (*d_off) cudaFree(*d_off);
    if (*d_ent) cudaFree(*d_ent);
    *d_off = nullptr;
    *d_ent = nullptr;
  }
  return cuda_status(err, "pair staging tables");
}

// Staging tables of candidate i, built the first time a pair kernel is
// selected (plan creation for the initial choice, else set_variant).
static int ensure_pair_tables(spp_dmt_plan* p, int i) {
  const Variant& v = variants()[p->cands[i]];
  if (!v.pairs || p->pair_off[i]) return SPP_OK;
  return pair_tables(p, p->delays_h.data(), v.DW, v.SLAB, slot_words(v, p->spans[i]),
                     &p->pair_off[i], &p->pair_ent[i]);
}

static void free_pair_tables(spp_dmt_plan* p) {
  for (int2* q : p->pair_off) if (q) cudaFree(q);
  for (int2* q : p->pair_ent) if (q) cudaFree(q);
  p->pair_off.clear();
  p->pair_ent.clear();
  if (p->d_pair_src) cudaFree(p->d_pair_src);
  p->d_pair_src = nullptr;
}

extern "C" {

int spp_dmt_plan_create(spp_dmt_plan** plan, int nbits, int bitorder, int64_t nchans,
                        int64_t nsamps_max, int64_t ndm, const int32_t* delays_host, int mode,
                        int out_kind, int acc) {
  if (!plan || !delays_host) return fail(SPP_ERR_ARG, "spp_dmt_plan_create: null pointer");
  *plan = nullptr;
  if (!valid_nbits(nbits)) return fail(SPP_ERR_ARG, "nbits must be 1, 2, 4, 8 or 32 (got %d)", nbits);
  if (nchans <= 0 || ndm <= 0 || nsamps_max <= 0 || nchans > INT32_MAX || ndm > INT32_MAX)
    return fail(SPP_ERR_ARG, "bad shape");
  if (nbits < 8 && (nchans * nbits) % 8 != 0)
    return fail(SPP_ERR_ARG, "nchans*nbits must be a multiple of 8");
  if (mode != SPP_MODE_DEDISPERSE && mode != SPP_MODE_ROLL) return fail(SPP_ERR_ARG, "bad mode");
  if (out_kind != SPP_OUT_F32 && out_kind != SPP_OUT_I32) return fail(SPP_ERR_ARG, "bad out_kind");
  if (out_kind == SPP_OUT_I32 && nbits == 32)
    return fail(SPP_ERR_ARG, "int32 output needs integer input");
  if (acc != SPP_ACC_F64 && acc != SPP_ACC_KAHAN32) return fail(SPP_ERR_ARG, "bad acc");
  if (bitorder != SPP_BITORDER_BIG && bitorder != SPP_BITORDER_LITTLE)
    return fail(SPP_ERR_ARG, "bad bitorder");
  spp_dmt_plan* p = new (std::nothrow) spp_dmt_plan();
  if (!p) return fail(SPP_ERR_ARG, "out of host memory");
  p->nbits = nbits; p->bitorder = bitorder; p->mode = mode; p->out_kind = out_kind; p->acc = acc;
  p->nchans = nchans; p->nsamps_max = nsamps_max; p->ndm = ndm;
  int32_t dmin = INT32_MAX, dmax = INT32_MIN;
  for (int64_t i = 0; i < ndm * nchans; ++i) {
    dmin = std::min(dmin, delays_host[i]);
    dmax = std::max(dmax, delays_host[i]);
  }
  p->dmin = dmin; p->dmax = dmax;
  p->maxabs = (int32_t)std::max<int64_t>(std::llabs(dmin), std::llabs(dmax));
  const int sign = plan_sign(p);
  p->omin = sign > 0 ? dmin : -dmax;
  p->omax = sign > 0 ? dmax : -dmin;
  if (mode == SPP_MODE_ROLL && p->maxabs >= nsamps_max) {
    delete p;
    return fail(SPP_ERR_DELAY, "roll mode needs |delay| < nsamps");
  }
  // candidates; the delay spread of DM tiles is computed once per tile height
  const auto& vs = variants();
  std::vector<std::pair<int, int32_t>> span_of_dw;
  auto tile_span = [&](int dw) -> int32_t {
    for (auto& e : span_of_dw)
      if (e.first == dw) return e.second;
    int32_t span = 0;
    std::vector<int32_t> mn(nchans), mx(nchans);
    for (int64_t d0 = 0; d0 < ndm; d0 += dw) {
      const int64_t d1 = std::min<int64_t>(ndm, d0 + dw);
      std::copy(delays_host + d0 * nchans, delays_host + (d0 + 1) * nchans, mn.begin());
      std::copy(mn.begin(), mn.end(), mx.begin());
      for (int64_t d = d0 + 1; d < d1; ++d) {
        const int32_t* row = delays_host + d * nchans;
        for (int64_t c = 0; c < nchans; ++c) {
          mn[c] = std::min(mn[c], row[c]);
          mx[c] = std::max(mx[c], row[c]);
        }
      }
      for (int64_t c = 0; c < nchans; ++c) span = std::max(span, mx[c] - mn[c]);
    }
    span_of_dw.emplace_back(dw, span);
    return span;
  };
  // Channel pairs (2-bit data): pair k = channels (2k, 2k+1) summed at the
  // relative offset r = o(2k+1) - o(2k), one row per (k, r) over all DMs
  // (at most 12 rows per channel, else the pair kernels are not offered).
  std::vector<int2> pair_src;
  if (nbits == 2) {
    const int64_t np = nchans / 2;
    std::vector<int32_t> rlo(np, INT32_MAX), rhi(np, INT32_MIN);
    for (int64_t d = 0; d < ndm; ++d) {
      const int32_t* row = delays_host + d * nchans;
      for (int64_t k = 0; k < np; ++k) {
        const int32_t r = sign * (row[2 * k + 1] - row[2 * k]);
        rlo[k] = std::min(rlo[k], r);
        rhi[k] = std::max(rhi[k], r);
      }
    }
    std::vector<int64_t> rbase(np);
    int64_t nrows = 0;
    for (int64_t k = 0; k < np; ++k) {
      rbase[k] = nrows;
      nrows += (int64_t)rhi[k] - rlo[k] + 1;
    }
    if (nrows <= 12 * nchans) {
      pair_src.resize(nrows);
      for (int64_t k = 0; k < np; ++k)
        for (int32_t r = rlo[k]; r <= rhi[k]; ++r)
          pair_src[rbase[k] + (r - rlo[k])] = make_int2((int)k, r);
      p->pair_rows.resize(ndm * np);
      for (int64_t d = 0; d < ndm; ++d) {
        const int32_t* row = delays_host + d * nchans;
        for (int64_t k = 0; k < np; ++k) {
          const int32_t r = sign * (row[2 * k + 1] - row[2 * k]);
          p->pair_rows[d * np + k] = (int32_t)(rbase[k] + (r - rlo[k]));
        }
      }
      p->nprows = nrows;
    }
  }
  // a pair kernel's stage holds 2 x slab rows: in every DM tile each pair
  // may use up to three distinct rows, and each slab's pairs together at
  // most 2 x slab
  std::vector<std::pair<int64_t, bool>> pairs_of_shape;
  auto pairs_fit = [&](int dw, int slab) -> bool {
    if (p->nprows == 0) return false;
    const int64_t key = (int64_t)dw << 16 | slab;
    for (auto& e : pairs_of_shape)
      if (e.first == key) return e.second;
    const int64_t np = nchans / 2;
    bool fit = true;
    for (int64_t d0 = 0; d0 < ndm && fit; d0 += dw) {
      const int64_t d1 = std::min<int64_t>(ndm, d0 + dw);
      int64_t used = 0;
      for (int64_t k = 0; k < np && fit; ++k) {
        int32_t u[3];
        int n = 0;
        for (int64_t d = d0; d < d1 && fit; ++d) {
          const int32_t r = p->pair_rows[d * np + k];
          bool seen = false;
          for (int i = 0; i < n; ++i) seen = seen || u[i] == r;
          if (seen) continue;
          if (n == 3) fit = false;
          else u[n++] = r;
        }
        used += n;
        if ((k + 1) % slab == 0 || k + 1 == np) {
          if (used > 2 * slab) fit = false;
          used = 0;
        }
      }
    }
    pairs_of_shape.emplace_back(key, fit);
    return fit;
  };
  for (int i = 0; i < (int)vs.size(); ++i) {
    const Variant& v = vs[i];
    if (v.nb != nbits || (nbits == 32 && v.acc != acc)) continue;
    if (v.pairs && !pairs_fit(v.DW, v.SLAB)) continue;
    if (ndm == 1 ? !v.single : v.single) continue;
    if (v.planes && nchans * ((1 << nbits) - 1) >= (1 << bit_levels(nbits))) continue;
    const int32_t span = tile_span(v.DW);
    if (slot_words(v, span) < 0) continue;  // fixed slot too narrow for this table
    if (smem_bytes(v, slot_words(v, span)) > kMaxSmem) continue;
    p->cands.push_back(i);
    p->spans.push_back(span);
  }
  if (p->cands.empty()) {
    delete p;
    return fail(SPP_ERR_UNSUPPORTED, "no kernel variant fits this delay table");
  }
  p->dpitch = nchans;
  cudaError_t e = cudaMalloc(&p->d_delays, sizeof(int32_t) * ndm * nchans);
  if (e != cudaSuccess) { delete p; return cuda_status(e, "plan cudaMalloc"); }
  e = cudaMemcpy(p->d_delays, delays_host, sizeof(int32_t) * ndm * nchans, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(p->d_delays); delete p; return cuda_status(e, "plan upload"); }
  bool use_pairs = false;
  for (int c : p->cands) use_pairs = use_pairs || vs[c].pairs;
  p->pair_off.assign(p->cands.size(), nullptr);
  p->pair_ent.assign(p->cands.size(), nullptr);
  if (use_pairs) {
    e = cudaMalloc(&p->d_pair_src, sizeof(int2) * pair_src.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_pair_src, pair_src.data(), sizeof(int2) * pair_src.size(),
                     cudaMemcpyHostToDevice);
    const int rc = cuda_status(e, "plan pair rows");
    if (rc != SPP_OK) {
      free_pair_tables(p);
      cudaFree(p->d_delays);
      delete p;
      return rc;
    }
    p->delays_h.assign(delays_host, delays_host + ndm * nchans);
  } else {
    p->pair_rows.clear();
    p->pair_rows.shrink_to_fit();
  }
  // without autotuning, start from the first fixed-slot pair kernel when the
  // table admits one (config 2: 17.1 ms against 22.1 ms for the first
  // per-channel kernel at 2^18 outputs) and its pair rows at nsamps_max stay
  // within kPairDefaultBytes (longer blocks keep the pair kernels for explicit
  // choice only: their rows grow with the block)
  constexpr int64_t kPairDefaultBytes = 16ll << 30;
  for (size_t i = 0; i < p->cands.size(); ++i) {
    const Variant& v = vs[p->cands[i]];
    if (!v.pairs || v.slot <= 0) continue;
    const int slot = slot_words(v, p->spans[i]);
    const Geometry g = geometry(v, nchans, nsamps_max, plan_nvalid(p, nsamps_max), p->omin,
                                p->omax, slot);
    if (p->nprows * 3 * g.pitch_w * 4 <= kPairDefaultBytes) p->cur = (int)i;
    break;
  }
  const int trc = ensure_pair_tables(p, p->cur);
  if (trc != SPP_OK) {
    free_pair_tables(p);
    cudaFree(p->d_delays);
    delete p;
    return trc;
  }
  *plan = p;
  return SPP_OK;
}

int spp_dmt_plan_destroy(spp_dmt_plan* p) {
  if (!p) return SPP_OK;
  int rc = SPP_OK;
  for (cudaEvent_t e : p->evpool) cudaEventDestroy(e);
  if (p->d_delays) rc = cuda_status(cudaFree(p->d_delays), "plan cudaFree");
  free_pair_tables(p);
  delete p;
  return rc;
}

int64_t spp_dmt_plan_nvalid(const spp_dmt_plan* p, int64_t nsamps) {
  if (!p) return -1;
  return std::max<int64_t>(0, plan_nvalid(p, nsamps));
}

int spp_dmt_plan_num_variants(const spp_dmt_plan* p) { return p ? (int)p->cands.size() : 0; }

int spp_dmt_plan_set_variant(spp_dmt_plan* p, int variant) {
  if (!p) return fail(SPP_ERR_ARG, "null plan");
  if (variant < 0 || variant >= (int)p->cands.size()) return fail(SPP_ERR_ARG, "bad variant %d", variant);
  const int rc = ensure_pair_tables(p, variant);
  if (rc != SPP_OK) return rc;
  p->cur = variant;
  return SPP_OK;
}

int spp_dmt_plan_describe(const spp_dmt_plan* p, int32_t* cfg) {
  if (!p || !cfg) return fail(SPP_ERR_ARG, "null pointer");
  const Variant& v = variants()[p->cands[p->cur]];
  const int slot = slot_words(v, p->spans[p->cur]);
  cfg[0] = v.nb | (v.planes << 8) | (v.pairs << 9); cfg[1] = v.R; cfg[2] = v.DW; cfg[3] = v.TW; cfg[4] = v.SLAB;
  cfg[5] = v.STAGES;
  cfg[6] = (int32_t)tile_T(v);
  cfg[7] = (int32_t)smem_bytes(v, slot);
  return SPP_OK;
}

static Geometry plan_geometry(const spp_dmt_plan* p, int64_t nsamps, int* slot) {
  const Variant& v = variants()[p->cands[p->cur]];
  *slot = slot_words(v, p->spans[p->cur]);
  return geometry(v, p->nchans, nsamps, plan_nvalid(p, nsamps), p->omin, p->omax, *slot);
}

// pair-sum rows follow the channel rows in the workspace
static int64_t pair_bytes(const spp_dmt_plan* p, const Geometry& g) {
  return variants()[p->cands[p->cur]].pairs ? p->nprows * 3 * g.pitch_w * 4 : 0;
}

int64_t spp_dmt_plan_workspace_bytes(const spp_dmt_plan* p, int64_t nsamps) {
  if (!p) return -1;
  int slot;
  Geometry g = plan_geometry(p, nsamps, &slot);
  return kStatusBytes + g.bytes + pair_bytes(p, g);
}

static int dmt_run(const spp_dmt_plan* p, const void* in, int64_t nsamps, void* out,
                   int64_t out_stride, int64_t out_start, uint8_t* ws, int64_t ws_bytes,
                   cudaStream_t st, const float* zd_bpass = nullptr,
                   const float* zd_chanwts = nullptr, double* zd_rows = nullptr) {
  int slot;
  Geometry g = plan_geometry(p, nsamps, &slot);
  if (g.nvalid <= 0) return SPP_OK;
  if (p->mode == SPP_MODE_ROLL && p->maxabs >= nsamps)
    return fail(SPP_ERR_DELAY, "roll mode needs |delay| < nsamps");
  if (-(int64_t)p->omin > nsamps)
    return fail(SPP_ERR_DELAY, "negative offset %d reaches before the block", p->omin);
  const int64_t pb = pair_bytes(p, g);
  if (ws_bytes < kStatusBytes + g.bytes + pb)
    return fail(SPP_ERR_SIZE, "workspace %lld B < required %lld B", (long long)ws_bytes,
                (long long)(kStatusBytes + g.bytes + pb));
  if (out_start < 0 || (p->ndm > 1 && out_stride < out_start + g.nvalid))
    return fail(SPP_ERR_SIZE, "out_stride %lld < out_start %lld + nvalid %lld",
                (long long)out_stride, (long long)out_start, (long long)g.nvalid);
  if (g.ntiles_t > 65535)
    return fail(SPP_ERR_UNSUPPORTED, "%lld time tiles exceed the grid limit", (long long)g.ntiles_t);
  const Variant& v = variants()[p->cands[p->cur]];
  void* planar = ws + kStatusBytes;
  spp_dmt_plan* pm = const_cast<spp_dmt_plan*>(p);
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  if (p->timing) {
    for (int i = 0; i < 3; ++i) {
      ev[i] = plan_event(pm);
      if (!ev[i]) return fail(SPP_ERR_CUDA, "cudaEventCreate failed");
    }
    cudaEventRecord(ev[0], st);
  }
  int rc = SPP_OK;
  if (zd_rows) {
    const unsigned blocks = (unsigned)ceil_div(nsamps, 32 * kRowSumWarps);
    k_row_sum_f64<<<blocks, 32 * kRowSumWarps, 0, st>>>(static_cast<const float*>(in), p->nchans, nsamps, zd_rows);
    rc = cuda_status(cudaGetLastError(), "zero-DM row sums");
    if (rc) return rc;
  }
  // float64 sums of float32 rows: the corner turn flags samples that are not
  // normal floats (word kSpecialWord of the status block, cleared here)
  uint32_t* special = nullptr;
  if (p->nbits == 32 && v.acc == SPP_ACC_F64) {
    special = reinterpret_cast<uint32_t*>(ws) + kSpecialWord;
    rc = cuda_status(cudaMemsetAsync(special, 0, 4, st), "special-value flag clear");
    if (rc) return rc;
  }
  rc = launch_corner_turn(p->nbits, in, p->bitorder, p->nchans, nsamps, g, planar, st, zd_rows,
                          zd_chanwts, zd_bpass, special);
  if (rc) return rc;
  if (v.pairs) {
    // pair-sum rows from the channel planes: one row per (pair, offset)
    uint32_t* pp = reinterpret_cast<uint32_t*>(ws + kStatusBytes + g.bytes);
    const int64_t gy = ceil_div(g.pitch_w, 4 * 256);
    if (gy > 65535 || p->nprows > INT32_MAX)
      return fail(SPP_ERR_UNSUPPORTED, "pair rows: %lld words x %lld rows", (long long)g.pitch_w,
                  (long long)p->nprows);
    k_pair_sums2<<<dim3((unsigned)p->nprows, (unsigned)gy), 256, 0, st>>>(
        static_cast<const uint32_t*>(planar), g.pitch_w, p->d_pair_src, pp);
    rc = cuda_status(cudaGetLastError(), "pair sums launch");
    if (rc) return rc;
    planar = pp;
  }
  if (p->timing) cudaEventRecord(ev[1], st);
  DmtArgs a{};
  a.planar = planar;
  a.pitch_w = g.pitch_w;
  a.halo = g.halo;
  a.nchans = (int32_t)p->nchans;
  a.delays = p->d_delays;
  a.dpitch = p->dpitch;
  a.ndm = (int32_t)p->ndm;
  a.sign = plan_sign(p);
  a.dlo = p->omin;
  a.dhi = p->omax;
  a.span_max = p->spans[p->cur];
  a.slot_w = slot;
  a.out = out;
  a.out_kind = p->out_kind;
  a.out_stride = out_stride;
  a.out_start = out_start;
  a.nvalid = g.nvalid;
  a.status = reinterpret_cast<uint32_t*>(ws);
  a.special = special;
  a.pair_off = p->pair_off[p->cur];
  a.pair_ent = p->pair_ent[p->cur];
  a.npairs = (int32_t)(p->nchans / 2);
  rc = launch_dmt(v, a, g.ntiles_t, p->ndm, st);
  if (rc) return rc;
  if (p->timing) cudaEventRecord(ev[2], st);
  return SPP_OK;
}

int spp_dmt_plan_timing(spp_dmt_plan* p, int enable) {
  if (!p) return fail(SPP_ERR_ARG, "null plan");
  p->timing = enable != 0;
  p->evused = 0;
  return SPP_OK;
}

int spp_dmt_plan_timing_read(spp_dmt_plan* p, double* ms_corner_turn, double* ms_dmt,
                             int32_t* nexec) {
  if (!p || !ms_corner_turn || !ms_dmt || !nexec) return fail(SPP_ERR_ARG, "null pointer");
  double a = 0.0, b = 0.0;
  const size_t n = p->evused / 3;
  for (size_t i = 0; i < n; ++i) {
    float x = 0.f, y = 0.f;
    int rc = cuda_status(cudaEventSynchronize(p->evpool[3 * i + 2]), "event sync");
    if (rc) return rc;
    rc = cuda_status(cudaEventElapsedTime(&x, p->evpool[3 * i], p->evpool[3 * i + 1]), "elapsed");
    if (rc) return rc;
    rc = cuda_status(cudaEventElapsedTime(&y, p->evpool[3 * i + 1], p->evpool[3 * i + 2]), "elapsed");
    if (rc) return rc;
    a += x;
    b += y;
  }
  *ms_corner_turn = a;
  *ms_dmt = b;
  *nexec = (int32_t)n;
  return SPP_OK;
}

int spp_dmt_execute(const spp_dmt_plan* p, const void* in, int64_t nsamps, void* out,
                    int64_t out_stride, int64_t out_start, void* workspace,
                    int64_t workspace_bytes, void* stream) {
  if (!p || !in || !out || !workspace) return fail(SPP_ERR_ARG, "spp_dmt_execute: null pointer");
  if (nsamps <= 0 || nsamps > p->nsamps_max)
    return fail(SPP_ERR_SIZE, "nsamps %lld outside (0, %lld]", (long long)nsamps, (long long)p->nsamps_max);
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return fail(SPP_ERR_ALIGN, "workspace must be 256-B aligned");
  return dmt_run(p, in, nsamps, out, out_stride, out_start, static_cast<uint8_t*>(workspace),
                 workspace_bytes, as_stream(stream));
}

int64_t spp_dmt_plan_zero_dm_workspace_bytes(const spp_dmt_plan* p, int64_t nsamps) {
  if (!p) return -1;
  return spp_dmt_plan_workspace_bytes(p, nsamps) + round_up(nsamps * 8, 256);
}

int spp_dmt_execute_zero_dm(const spp_dmt_plan* p, const float* in, int64_t nsamps,
                            const float* bpass, const float* chanwts, void* out,
                            int64_t out_stride, int64_t out_start, void* workspace,
                            int64_t workspace_bytes, void* stream) {
  if (!p || !in || !bpass || !chanwts || !out || !workspace) return fail(SPP_ERR_ARG, "null pointer");
  if (p->nbits != 32) return fail(SPP_ERR_UNSUPPORTED, "zero-DM fusion needs float32 input");
  if (nsamps <= 0 || nsamps > p->nsamps_max) return fail(SPP_ERR_SIZE, "nsamps out of range");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return fail(SPP_ERR_ALIGN, "workspace must be 256-B aligned");
  const int64_t need = spp_dmt_plan_zero_dm_workspace_bytes(p, nsamps);
  if (workspace_bytes < need) return fail(SPP_ERR_SIZE, "workspace %lld < %lld", (long long)workspace_bytes, (long long)need);
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  double* rows = reinterpret_cast<double*>(ws + spp_dmt_plan_workspace_bytes(p, nsamps));
  return dmt_run(p, in, nsamps, out, out_stride, out_start, ws, workspace_bytes, as_stream(stream),
                 bpass, chanwts, rows);
}

// --- end-to-end from host buffers ------------------------------------------------
static int64_t host_row_bytes(const spp_dmt_plan* p) {
  return p->nbits == 32 ? p->nchans * 4 : p->nchans * p->nbits / 8;
}

struct HostLayout {
  int64_t in_rows, in_bytes, out_bytes, run_bytes, set_bytes;
};

static HostLayout host_layout(const spp_dmt_plan* p, int64_t block) {
  HostLayout h{};
  h.in_rows = block + p->maxabs;
  h.in_bytes = round_up(h.in_rows * host_row_bytes(p), 256);
  h.out_bytes = round_up(p->ndm * block * 4, 256);
  h.run_bytes = round_up(spp_dmt_plan_workspace_bytes(p, h.in_rows), 256);
  h.set_bytes = h.in_bytes + h.out_bytes + h.run_bytes;
  return h;
}

// Host streaming keeps this many block buffer sets (and streams) in flight:
// copies in, DM kernel and copies out of consecutive blocks overlap.
constexpr int kHostSets = 3;

int64_t spp_dmt_host_workspace_bytes(const spp_dmt_plan* p, int64_t block_nsamps) {
  if (!p || block_nsamps <= 0) return -1;
  return kStatusBytes + kHostSets * host_layout(p, block_nsamps).set_bytes;
}

int spp_dmt_execute_host(const spp_dmt_plan* p, const void* in_host, int64_t nsamps,
                         void* out_host, int64_t out_stride, int64_t block_nsamps,
                         void* workspace, int64_t workspace_bytes) {
  if (!p || !in_host || !out_host || !workspace) return fail(SPP_ERR_ARG, "null pointer");
  if (p->mode != SPP_MODE_DEDISPERSE || p->omin < 0)
    return fail(SPP_ERR_UNSUPPORTED, "host streaming needs dedisperse mode and delays >= 0");
  if (block_nsamps <= 0) return fail(SPP_ERR_ARG, "block_nsamps <= 0");
  const int64_t nvalid = plan_nvalid(p, nsamps);
  if (nvalid <= 0) return SPP_OK;
  if (out_stride < nvalid) return fail(SPP_ERR_SIZE, "out_stride < nvalid");
  const HostLayout h = host_layout(p, block_nsamps);
  if (h.in_rows > p->nsamps_max)
    return fail(SPP_ERR_SIZE, "block + max delay (%lld) exceeds plan nsamps_max", (long long)h.in_rows);
  if (workspace_bytes < kStatusBytes + kHostSets * h.set_bytes)
    return fail(SPP_ERR_SIZE, "workspace too small");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return fail(SPP_ERR_ALIGN, "workspace must be 256-B aligned");
  uint8_t* ws = static_cast<uint8_t*>(workspace);
  cudaStream_t s[kHostSets];
  int rc = SPP_OK;
  for (int i = 0; i < kHostSets; ++i) {
    rc = cuda_status(cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking), "stream create");
    if (rc) {
      for (int j = 0; j < i; ++j) cudaStreamDestroy(s[j]);
      return rc;
    }
  }
  const int64_t rb = host_row_bytes(p);
  const int64_t es = 4;
  const int64_t nblocks = ceil_div(nvalid, block_nsamps);
  // each buffer set's run workspace starts with the device status words of
  // the kernels it hosts: cleared here, read back once everything finished
  for (int k = 0; k < kHostSets && rc == SPP_OK; ++k)
    rc = cuda_status(cudaMemsetAsync(ws + kStatusBytes + k * h.set_bytes + h.in_bytes + h.out_bytes,
                                     0, 16, s[k]),
                     "status clear");
  for (int64_t b = 0; b < nblocks && rc == SPP_OK; ++b) {
    const int k = (int)(b % kHostSets);
    uint8_t* set = ws + kStatusBytes + k * h.set_bytes;
    uint8_t* d_in = set;
    uint8_t* d_out = set + h.in_bytes;
    uint8_t* d_run = set + h.in_bytes + h.out_bytes;
    const int64_t t0 = b * block_nsamps;
    const int64_t nout = std::min(block_nsamps, nvalid - t0);
    const int64_t rows = nout + p->maxabs;
    rc = cuda_status(cudaMemcpyAsync(d_in, static_cast<const uint8_t*>(in_host) + t0 * rb,
                                     rows * rb, cudaMemcpyHostToDevice, s[k]), "H2D");
    if (rc) break;
    rc = dmt_run(p, d_in, rows, d_out, nout, 0, d_run, h.run_bytes, s[k]);
    if (rc) break;
    rc = cuda_status(cudaMemcpy2DAsync(static_cast<uint8_t*>(out_host) + t0 * es, out_stride * es,
                                       d_out, nout * es, nout * es, p->ndm,
                                       cudaMemcpyDeviceToHost, s[k]), "D2H");
  }
  for (int i = 0; i < kHostSets; ++i) {
    int r2 = cuda_status(cudaStreamSynchronize(s[i]), "stream sync");
    if (!rc) rc = r2;
    cudaStreamDestroy(s[i]);
  }
  for (int k = 0; k < kHostSets && rc == SPP_OK; ++k) {
    uint32_t words[4] = {0, 0, 0, 0};
    rc = cuda_status(cudaMemcpy(words, ws + kStatusBytes + k * h.set_bytes + h.in_bytes + h.out_bytes,
                                16, cudaMemcpyDeviceToHost),
                     "status copy");
    if (rc == SPP_OK && words[0] != 0)
      rc = fail(SPP_ERR_DEVICE, "device status 0x%x (block %u, detail 0x%x)", words[0], words[1],
                words[2]);
  }
  return rc;
}

}  // extern "C"
