// Seeded synthetic filterbank generators for the benchmark workloads.
// Counter-based: value i depends only on (seed, i) through the SplitMix64
// finaliser (Steele, Lea & Flood 2014), so any slice can be regenerated on
// the host bit for bit (sigpyproc3_b200/synth.py holds the numpy twins).
#include <algorithm>

#include "spp_common.cuh"

namespace spp {

static inline cudaStream_t st_of(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__device__ __forceinline__ uint64_t mix64(uint64_t seed, uint64_t i) {
  uint64_t z = (seed << 40) ^ i;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void k_uniform_bytes(uint8_t* __restrict__ out, int64_t start, int64_t n, uint64_t seed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (uint8_t)(mix64(seed, (uint64_t)(start + i)) & 0xFFu);
}

struct Thresholds {
  uint32_t t[255];
};

__global__ void k_gauss_u8(uint8_t* __restrict__ out, int64_t start, int64_t n, uint64_t seed,
                           const Thresholds th) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(mix64(seed, (uint64_t)(start + i)) >> 32);
    // number of thresholds <= u (upper bound binary search over 255 entries)
    int lo = 0, hi = 255;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (th.t[mid] <= u) lo = mid + 1; else hi = mid;
    }
    out[i] = (uint8_t)lo;
  }
}

// Box-Muller normal deviates (device only; libm-dependent low bits).
__global__ void k_gauss_f32(float* __restrict__ out, int64_t start, int64_t n, uint64_t seed,
                            float mean, float stdv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = mix64(seed, (uint64_t)(start + i));
    const float u1 = ((float)(h >> 40) + 1.0f) * (1.0f / 16777217.0f);        // (0, 1]
    const float u2 = (float)((h >> 16) & 0xFFFFFFu) * (1.0f / 16777216.0f);   // [0, 1)
    const float r = sqrtf(-2.0f * logf(u1));
    out[i] = mean + stdv * r * cospif(2.0f * u2);
  }
}

// Adds +1 (saturating at the field maximum) to the packed field of channel c
// for rows start_rows[c] .. start_rows[c] + width - 1 (rows outside the block
// are skipped).  Fields in the same byte are updated with atomicCAS on the
// containing 32-bit word.
__global__ void k_pulse_packed(uint8_t* __restrict__ raw, int64_t nchans, int64_t nsamps, int nbits,
                               int big, const int64_t* __restrict__ start_rows, int width) {
  const int64_t total = nchans * width;
  const uint32_t fmax = (1u << nbits) - 1u;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = idx / width, k = idx - c * width;
    const int64_t row = start_rows[c] + k;
    if (row < 0 || row >= nsamps) continue;
    const int64_t bit = (row * nchans + c) * nbits;
    const int64_t byte = bit >> 3;
    const int per = 8 / nbits, p = (int)(c % per);
    const int sh_in_byte = big ? (8 - (p + 1) * nbits) : (p * nbits);
    uint32_t* word = reinterpret_cast<uint32_t*>(raw + (byte & ~int64_t(3)));
    const int sh = (int)(byte & 3) * 8 + sh_in_byte;
    uint32_t old = *word, assumed;
    do {
      assumed = old;
      const uint32_t f = (assumed >> sh) & fmax;
      if (f == fmax) break;
      old = atomicCAS(word, assumed, assumed + (1u << sh));
    } while (old != assumed);
  }
}

// Self-test of the bounded-wait path: an mbarrier expecting two arrivals gets
// one, so its phase never completes; the wait gives up after limit_ns and
// records SPP_DEV_TIMEOUT in the status word.
__global__ void k_wait_selftest(uint32_t* status, uint64_t limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 2);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive(&bar);
    mbar_wait_ns(&bar, 0, status, limit_ns);
  }
  __syncthreads();
}

}  // namespace spp

using namespace spp;

extern "C" {

int spp_synth_uniform_bytes(uint8_t* out, int64_t start, int64_t n, uint64_t seed, void* stream) {
  if (!out || n < 0) return fail(SPP_ERR_ARG, "bad arguments");
  if (n == 0) return SPP_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 64);
  k_uniform_bytes<<<blocks, 256, 0, st_of(stream)>>>(out, start, n, seed);
  return cuda_status(cudaGetLastError(), "synth launch");
}

int spp_synth_gauss_u8(uint8_t* out, int64_t start, int64_t n, uint64_t seed,
                       const uint32_t* thresholds_host, void* stream) {
  if (!out || !thresholds_host || n < 0) return fail(SPP_ERR_ARG, "bad arguments");
  if (n == 0) return SPP_OK;
  Thresholds th;
  for (int i = 0; i < 255; ++i) th.t[i] = thresholds_host[i];
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 64);
  k_gauss_u8<<<blocks, 256, 0, st_of(stream)>>>(out, start, n, seed, th);
  return cuda_status(cudaGetLastError(), "synth launch");
}

int spp_synth_gauss_f32(float* out, int64_t start, int64_t n, uint64_t seed, float mean,
                        float stdv, void* stream) {
  if (!out || n < 0) return fail(SPP_ERR_ARG, "bad arguments");
  if (n == 0) return SPP_OK;
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 64);
  k_gauss_f32<<<blocks, 256, 0, st_of(stream)>>>(out, start, n, seed, mean, stdv);
  return cuda_status(cudaGetLastError(), "synth launch");
}

int spp_selftest_wait_timeout(uint32_t* status, uint64_t limit_ns, void* stream) {
  if (!status) return fail(SPP_ERR_ARG, "null status");
  if (limit_ns > 1000000000ull) return fail(SPP_ERR_ARG, "limit above one second");
  k_wait_selftest<<<1, 32, 0, st_of(stream)>>>(status, limit_ns);
  return cuda_status(cudaGetLastError(), "self-test launch");
}

int spp_synth_pulse_packed(uint8_t* raw, int64_t nchans, int64_t nsamps, int nbits, int bitorder,
                           const int64_t* start_rows, int width, void* stream) {
  if (!raw || !start_rows || width <= 0) return fail(SPP_ERR_ARG, "bad arguments");
  if (nbits != 1 && nbits != 2 && nbits != 4 && nbits != 8) return fail(SPP_ERR_ARG, "bad nbits");
  if ((reinterpret_cast<uintptr_t>(raw) & 3) != 0) return fail(SPP_ERR_ALIGN, "raw must be 4-B aligned");
  if (((nchans * nsamps * nbits) / 8) % 4 != 0) return fail(SPP_ERR_SIZE, "raw size must be a multiple of 4 bytes");
  const unsigned blocks = (unsigned)std::min<int64_t>(ceil_div(nchans * width, 256), 148 * 64);
  k_pulse_packed<<<blocks, 256, 0, st_of(stream)>>>(raw, nchans, nsamps, nbits,
                                                    bitorder == SPP_BITORDER_BIG, start_rows, width);
  return cuda_status(cudaGetLastError(), "synth launch");
}

}  // extern "C"
