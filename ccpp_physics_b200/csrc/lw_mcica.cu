// lw_mcica.cu -- McICA sub-column cloud generator on the GPU, bit-exact.
//
// Restates mcica_subcol (physics/Radiation/RRTMG/radlw_main.F90, RLM:1847-
// 2107) with the GFS Mersenne twister of physics/Radiation/
// mersenne_twister.f (random_setseed_t MT:285-299, random_number_t
// MT:330-372).  One warp owns one cloudy column:
//   * seeding mt(i) = 69069^i * seed (mod 2^32) is one multiply per word
//     with a table of powers of 69069 in constant memory;
//   * each twist of the 624-word state runs in three dependency phases
//     (words 0..226 from old words, 227..453 and 454..622 from words
//     already updated, then word 623), 32 words per lane step;
//   * for max-random overlap (iovr=1) the random array is g-point major
//     (rand2d index (n-1)*nlay+k, RLM:1935-1941), so each g-point's walk
//     reads a contiguous run of the stream.  Lanes own g-points, 32 at a
//     time; the stream is generated into a per-warp ring buffer just ahead
//     of the 32 walks that read it.
// Integer arithmetic is exact; the u32 -> real conversion (u/(2^32-1)) and
// the FP64 comparisons/products of the walk are IEEE operations, so the
// sub-column flags equal the Fortran's bit for bit.
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "lw_common.cuh"

namespace lw {

__device__ __constant__ uint32_t c_pow69069[624];

constexpr uint32_t kMata = 0x9908B0DFu, kUmask = 0x80000000u, kLmask = 0x7FFFFFFFu;
constexpr uint32_t kTmaskB = 0x9D2C5680u, kTmaskC = 0xEFC60000u;

__device__ __forceinline__ uint32_t mt_word(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t y = (a & kUmask) | (b & kLmask);
  return c ^ (y >> 1) ^ ((y & 1u) ? kMata : 0u);
}
__device__ __forceinline__ uint32_t temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & kTmaskB;
  y ^= (y << 15) & kTmaskC;
  y ^= y >> 18;
  return y;
}

// One twist of the warp's state mt[624] (MT:341-356), parallel over lanes.
__device__ void twist(uint32_t* mt, int lane) {
  // phase A: kk = 0..226 reads mt[kk], mt[kk+1] (old), mt[kk+397] (old)
  for (int base = 0; base < 227; base += 32) {
    int kk = base + lane;
    uint32_t v = 0;
    if (kk < 227) v = mt_word(mt[kk], mt[kk + 1], mt[kk + 397]);
    __syncwarp();
    if (kk < 227) mt[kk] = v;
    __syncwarp();
  }
  // phase B1: kk = 227..453 reads mt[kk-227] (new, from phase A)
  for (int base = 227; base < 454; base += 32) {
    int kk = base + lane;
    uint32_t v = 0;
    if (kk < 454) v = mt_word(mt[kk], mt[kk + 1], mt[kk - 227]);
    __syncwarp();
    if (kk < 454) mt[kk] = v;
    __syncwarp();
  }
  // phase B2: kk = 454..622 reads mt[kk-227] (new, from phase B1)
  for (int base = 454; base < 623; base += 32) {
    int kk = base + lane;
    uint32_t v = 0;
    if (kk < 623) v = mt_word(mt[kk], mt[kk + 1], mt[kk - 227]);
    __syncwarp();
    if (kk < 623) mt[kk] = v;
    __syncwarp();
  }
  // phase C: kk = 623 with mt[0] and mt[396] (both new)
  if (lane == 0) mt[623] = mt_word(mt[623], mt[0], mt[396]);
  __syncwarp();
}

// u / (2^32 - 1), correctly rounded, without a division (the GFS twister's
// harvest = real(y) / (2**32 - 1), mersenne_twister.f:362-369, for the
// unsigned value u of y).  1/(2^32-1) = (2^32+1)/(2^64-1), so the quotient
// is m * 2^-64 * (1 + 2^-64 + ...) with the 64-bit integer
// m = u * (2^32 + 1) = (u << 32) | u.  One FMA gives RN(m * 2^-64) exactly;
// the true quotient lies strictly above m * 2^-64 (for u > 0) but within one
// unit of m's last bit, so the two round alike except when m's discarded
// bits are exactly one half: then the quotient must round up, which ties-to-
// even misses when the kept last bit is 0.  m has 32 + L significant bits
// (L = bit length of u), so d = L - 21 bits are discarded, all from the low
// word, i.e. the low d bits of u.
__device__ __forceinline__ double u32_unit(uint32_t u) {
  const double a = (double)u * 0x1p-32;   // exact
  double r = fma(a, 0x1p-32, a);          // RN(m * 2^-64)
  const int d = (32 - __clz(u)) - 21;
  if (d >= 1) {
    const uint32_t half = 1u << (d - 1);
    if ((u & ((half << 1) - 1u)) == half && ((u >> d) & 1u) == 0u)
      r = __longlong_as_double(__double_as_longlong(r) + 1);
  }
  return r;
}

struct McicaArgs {
  int nlay, nw, iovr, isubclw, top_at_1;
  int cap;        // ring capacity in words
};

// Per-warp shared memory: mt[624], clear[nlay] = 1 - cldf (double), ring[cap].
__host__ __device__ inline size_t mcica_warp_bytes(int nlay, int cap) {
  return 624 * 4 + ((nlay * 8 + 15) & ~15) + (size_t)cap * 4 + 16;
}

constexpr int kMcicaWarps = 5;   // 5 warps x 22 KB (127 layers): two CTAs, ten warps per SM

__global__ void __launch_bounds__(32 * kMcicaWarps)
lw_mcica_kernel(const Block* __restrict__ blocks, int nblocks, const Block b0, int ncols, McicaArgs a,
                const double* __restrict__ cldf_dev, const int32_t* __restrict__ seed_dev, int dev_ld,
                uint32_t* __restrict__ bits) {
  extern __shared__ __align__(16) char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const size_t wbytes = mcica_warp_bytes(a.nlay, a.cap);
  char* my = smem_raw + wbytes * wib;
  uint32_t* mt = reinterpret_cast<uint32_t*>(my);
  double* clr = reinterpret_cast<double*>(my + 624 * 4);   // 1 - cldf(k), used by every test of the walk
  uint32_t* ring = reinterpret_cast<uint32_t*>(my + 624 * 4 + ((a.nlay * 8 + 15) & ~15));
  const int nlay = a.nlay, nlp1 = nlay + 1;
  const int warps_total = gridDim.x * (blockDim.x >> 5);

  for (int c = blockIdx.x * (blockDim.x >> 5) + wib; c < ncols; c += warps_total) {
    __syncwarp();
    int32_t seed;
    bool any = false;
    if (nblocks > 0) {
      // layer cloud fraction in internal (surface-first) order, floored as
      // in cldprop (RLM:1805-1811); lcf1 test of the driver (RLM:1070-1076)
      const Block& B = (nblocks == 1) ? b0 : blocks[find_block(blocks, nblocks, c)];
      const int i = c - B.col0;
      for (int k = lane; k < nlay; k += 32) {
        int r = a.top_at_1 ? nlp1 - (k + 1) - 1 : k;
        double cf = B.in[F_CLDCF][i + (size_t)B.ld * r];
        any |= cf > 1.0e-6;
        clr[k] = 1.0 - ((cf < 2.2250738585072014e-308) ? 0.0 : cf);
      }
      seed = (a.isubclw == 1) ? 140 + (i + 1) : B.icseed[i];   // RLM:765-773
    } else {
      for (int k = lane; k < nlay; k += 32) {
        clr[k] = 1.0 - cldf_dev[c + (size_t)dev_ld * k];
      }
      any = true;
      seed = seed_dev[c];
    }
    if (!__any_sync(0xffffffffu, any)) continue;   // clear column: no draws
    // random_setseed_t: mt(0)=seed (0 -> 4357), mt(i) = 69069*mt(i-1)
    uint32_t s0 = (uint32_t)(seed == 0 ? 4357 : seed);
    for (int n = lane; n < 624; n += 32) mt[n] = s0 * c_pow69069[n];
    __syncwarp();

    uint32_t* out = bits + (size_t)c * NGPT * a.nw;
    if (a.iovr == 2) {
      // maximum overlap: one draw per g-point, the same at every layer (RLM:1981-1993)
      twist(mt, lane);
      for (int n = lane; n < NGPT; n += 32) {
        double r = u32_unit(temper(mt[n]));
        for (int w = 0; w < a.nw; ++w) {
          uint32_t word = 0;
          for (int b = 0; b < 32; ++b) {
            int k = w * 32 + b;
            if (k < nlay && r >= clr[k]) word |= 1u << b;
          }
          out[n * a.nw + w] = word;
        }
      }
      continue;
    }
    // random (iovr=0) and maximum-random (iovr=1): stream position n*nlay+k
    const int cap = a.cap;
    long gen_end = 0;          // stream positions generated so far
    for (int n0 = 0; n0 < NGPT; n0 += 32) {
      const int n1 = min(n0 + 32, NGPT);
      const long need = (long)n1 * nlay;
      while (gen_end < need) {
        twist(mt, lane);
        int p = (int)(gen_end % cap);
        for (int j = lane; j < 624; j += 32) {
          int q = p + j;
          if (q >= cap) q -= cap;
          ring[q] = temper(mt[j]);
        }
        gen_end += 624;
        __syncwarp();
      }
      const int n = n0 + lane;
      if (n < n1) {
        int q = (int)(((long)n * nlay) % cap);
        double cdf = 0.0;
        uint32_t word = 0;
        for (int k = 0; k < nlay; ++k) {
          double r = u32_unit(ring[q]);
          if (++q == cap) q = 0;
          if (k == 0 || a.iovr == 0) {
            cdf = r;
          } else {
            double tem1 = clr[k - 1];              // max-random walk (RLM:1949-1960)
            cdf = (cdf > tem1) ? cdf : r * tem1;
          }
          if (cdf >= clr[k]) word |= 1u << (k & 31);   // RLM:2097-2103
          if ((k & 31) == 31 || k == nlay - 1) {
            out[n * a.nw + (k >> 5)] = word;
            word = 0;
          }
        }
      }
      __syncwarp();
    }
  }
}

// host side ------------------------------------------------------------------

int mcica_ring_capacity(int nlay) { return ((32 * nlay + 624 + 31) / 32) * 32; }

cudaError_t mcica_prepare(int max_smem) {
  return cudaFuncSetAttribute(lw_mcica_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
}

cudaError_t mcica_upload_powers() {
  static uint32_t pw[624];
  pw[0] = 1u;
  for (int i = 1; i < 624; ++i) pw[i] = pw[i - 1] * 69069u;
  return cudaMemcpyToSymbol(c_pow69069, pw, sizeof(pw));
}

cudaError_t mcica_launch(const Block* blocks, int nblocks, const Block& b0, int ncols, int nlay, int iovr, int isubclw,
                         int top_at_1, const double* cldf_dev, const int32_t* seed_dev, int dev_ld,
                         uint32_t* bits, int num_sms, cudaStream_t st) {
  McicaArgs a;
  a.nlay = nlay;
  a.nw = (nlay + 31) / 32;
  a.iovr = iovr;
  a.isubclw = isubclw;
  a.top_at_1 = top_at_1;
  a.cap = mcica_ring_capacity(nlay);
  const int wpb = kMcicaWarps;
  size_t smem = mcica_warp_bytes(nlay, a.cap) * wpb;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lw_mcica_kernel, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  int grid = min((ncols + wpb - 1) / wpb, num_sms * per_sm);
  if (grid < 1) return cudaSuccess;
  lw_mcica_kernel<<<grid, wpb * 32, smem, st>>>(blocks, nblocks, b0, ncols, a, cldf_dev, seed_dev, dev_ld, bits);
#if LW_DEBUG_CHECKS
  {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { fprintf(stderr, "lw debug: mcica kernel failed\n"); return e; }
  }
#endif
  return cudaGetLastError();
}

}  // namespace lw
