// lw_mcica.cu -- McICA sub-column cloud generator on the GPU, bit-exact.
//
// Restates mcica_subcol (physics/Radiation/RRTMG/radlw_main.F90, RLM:1847-
// 2107) with the GFS Mersenne twister of physics/Radiation/
// mersenne_twister.f (random_setseed_t MT:285-299, random_number_t
// MT:330-372).  One warp owns one cloudy column:
//   * seeding mt(i) = 69069^i * seed (mod 2^32) is one multiply per word
//     with a table of powers of 69069 in constant memory;
//   * the stream lives in shared memory as its raw (untempered) sequence; a
//     twist appends the next 624 words in place in three dependency phases
//     (words 0..226 from the previous block, 227..453 and 454..622 from
//     words 227 back, then word 623), one barrier each;
//   * for max-random overlap (iovr=1) the random array is g-point major
//     (rand2d index (n-1)*nlay+k, RLM:1935-1941), so each g-point's walk
//     reads a contiguous run of the stream.  Lanes own g-points, 28 at a
//     time; the sequence ring holds one round's draws and the twist history.
// Integer arithmetic is exact; the u32 -> real conversion (u/(2^32-1)) and
// the FP64 comparisons/products of the walk are IEEE operations, so the
// sub-column flags equal the Fortran's bit for bit.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "lw_common.cuh"
#include "lw_launch.h"

namespace lw {

__device__ __constant__ uint32_t c_pow69069[624];

constexpr uint32_t kMata = 0x9908B0DFu, kUmask = 0x80000000u, kLmask = 0x7FFFFFFFu;
constexpr uint32_t kTmaskB = 0x9D2C5680u, kTmaskC = 0xEFC60000u;
// untempered word whose tempering is 2^32 - 1 (the only draw equal to 1)
constexpr uint32_t kRawAllOnes = 0x12DD9BB3u;

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

// Appends the next 624 sequence words to the ring at position jp (a
// multiple of 624; the previous block sits just before it, cyclically)
// (MT:341-356): words 0..226 of the block from the previous block, 227..453
// and 454..622 from words 227 back in this block, 623 from x_{j-1}, x_j and
// x_{j+396}; one barrier per dependency phase.
// With HIT, also returns whether this lane wrote the one word that tempers to
// 2^32 - 1 (kRawAllOnes).
template <bool HIT = false>
__device__ bool twist_ring(uint32_t* ring, int cap, int jp, int lane) {
  const uint32_t* o = ring + ((jp == 0 ? cap : jp) - 624);
  uint32_t* w = ring + jp;
  bool hit = false;
  // fully unrolled, so each phase's shared-memory loads issue together
#pragma unroll
  for (int t = lane; t < 227; t += 32) {
    w[t] = mt_word(o[t], o[t + 1], o[t + 397]);
    if (HIT) hit |= w[t] == kRawAllOnes;
  }
  __syncwarp();
#pragma unroll
  for (int t = 227 + lane; t < 454; t += 32) {
    w[t] = mt_word(o[t], o[t + 1], w[t - 227]);
    if (HIT) hit |= w[t] == kRawAllOnes;
  }
  __syncwarp();
#pragma unroll
  for (int t = 454 + lane; t < 624; t += 32) {
    w[t] = mt_word(o[t], (t == 623) ? w[0] : o[t + 1], w[t - 227]);
    if (HIT) hit |= w[t] == kRawAllOnes;
  }
  __syncwarp();
  return hit;
}

struct McicaArgs {
  int nlay, nw, iovr, isubclw, top_at_1;
  int cap;        // ring capacity in words
  McicaStage st;  // stage entry point inputs (blocks == nullptr)
};

// One twister stream kept as a sequence ring of two blocks (1248 words;
// sequence index s at ring[s mod 1248], draw p = tempered x_{624+p}).  The
// reader tracks its next sequence index s, its ring position, and how far
// the sequence has been generated.
constexpr int kTwoSetRing = 1248;
struct TwoSetStream {
  int s;      // sequence index of the next draw
  int pos;    // s mod 1248
  int gen;    // sequence indices generated so far (a multiple of 624)
};

// The next 140 draws (one layer of a layer-major stream, RLM:2006-2024);
// lane gets the tempered words of g-points n = lane + 32 j (j < 5).  Blocks
// are appended as the reads advance; the block a new one overwrites was read
// before the barrier.
__device__ __forceinline__ void layer_draws(uint32_t* ring, TwoSetStream& st, int lane, uint32_t (&d)[5]) {
  if (st.gen < st.s + NGPT) {
    __syncwarp();
    do {
      twist_ring(ring, kTwoSetRing, (st.gen / 624) & 1 ? 624 : 0, lane);
      st.gen += 624;
    } while (st.gen < st.s + NGPT);
  }
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const int n = lane + 32 * j;
    int q = st.pos + n;
    if (q >= kTwoSetRing) q -= kTwoSetRing;
    d[j] = (n < NGPT) ? temper(ring[q]) : 0u;
  }
  st.s += NGPT;
  st.pos += NGPT;
  if (st.pos >= kTwoSetRing) st.pos -= kTwoSetRing;
}

// The draw conversion h(u) = u / (2^32 - 1) (u32_unit) is strictly
// increasing (consecutive u differ by 2^-32, far above a double's spacing),
// so every comparison of a draw with a per-layer value x is a comparison of
// the tempered word u with an exact integer threshold:
//   h(u) >= x  <=>  u >= umin_ge(x),   h(u) < x  <=>  u < ulim_lt(x),
//   h(u) <= x  <=>  u <= umax_le(x).
// Thresholds are 64-bit: 2^32 / -1 / 0 mean that no word qualifies (x above
// 1, below 0, or NaN, for which every comparison is false).  x (2^32 - 1) is
// within one unit of the threshold, so a few exact steps settle it.
__device__ long long umin_ge(double x) {
  if (x <= 0.0) return 0;
  if (!(x <= 1.0)) return 4294967296LL;
  long long u = (long long)(x * 4294967295.0);
  if (u > 4294967295LL) u = 4294967295LL;
  for (int it = 0; it < 8 && u > 0 && u32_unit((uint32_t)(u - 1)) >= x; ++it) --u;
  for (int it = 0; it < 8 && u <= 4294967295LL && u32_unit((uint32_t)u) < x; ++it) ++u;
  return u;
}
__device__ long long ulim_lt(double x) { return (x != x) ? 0 : umin_ge(x); }
__device__ long long umax_le(double x) {
  if (!(x >= 0.0)) return -1;
  if (x >= 1.0) return 4294967295LL;
  long long u = (long long)(x * 4294967295.0);   // smallest u with h(u) > x, minus one
  for (int it = 0; it < 8 && u > 0 && u32_unit((uint32_t)(u - 1)) > x; ++it) --u;
  for (int it = 0; it < 8 && u32_unit((uint32_t)u) <= x; ++it) ++u;
  return u - 1;
}

// Overlaps built from two layer-major random sets (RLM:1995-2091):
//   iovr = 3, decorrelation length: top-down, layer k keeps the value of layer
//     k+1 when set2(k) <= fac_lcf(k+1), else its own set-1 draw;
//   iovr = 4/5, exponential / exponential-random: bottom-up, layer k keeps the
//     value of layer k-1 when set2(k) < alpha(k), else its own draw.
// Set 1 is stream positions [0, 140 nlay), set 2 the next 140 nlay; two
// twister states walk them in lockstep, layer by layer, surface first.  The
// top-down rule is evaluated bottom-up: a layer's value is the set-1 draw of
// the nearest layer at or above it whose link to the layer above is broken
// (the top layer always is), so each g-point keeps the run of layers still
// waiting for that draw and resolves it when the break arrives.
// The walk runs on tempered words against integer thresholds (above):
// clr_t[k] = umin_ge(1 - cldf(k)) for the cloud test (RLM:2097-2103), and
// aux_t[k] = umax_le(fac_lcf(k)) (iovr 3, 0-based, aux_t[0] unused) or
// ulim_lt(alpha(k)) (iovr 4, 5).
__device__ void mcica_two_set(uint32_t* mtA, uint32_t* mtB, const long long* clr_t, const long long* aux_t,
                              const long long* srt, const uint32_t* pm, int nlay, int iovr, uint32_t s0, int nw,
                              uint32_t* out, int lane) {
  for (int n = lane; n < 624; n += 32) {
    const uint32_t v = s0 * c_pow69069[n];
    mtA[n] = v;
    mtB[n] = v;
  }
  __syncwarp();
  // set 2 starts at draw 140 nlay of the same stream: its first layer_draws
  // call appends blocks up to there
  const int P0 = NGPT * nlay;
  TwoSetStream sa{624, 624, 624}, sb{624 + P0, (624 + P0) % kTwoSetRing, 624};
  uint32_t cdf[5], c1[5], c2[5];
  uint32_t word[5] = {0u, 0u, 0u, 0u, 0u};
  int start[5] = {0, 0, 0, 0, 0}, wi[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < nlay; ++k) {
    layer_draws(mtA, sa, lane, c1);
    layer_draws(mtB, sb, lane, c2);
    if (iovr == 3) {
      const bool top = (k == nlay - 1);
      const long long fk = top ? 0 : aux_t[k + 1];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const int n = lane + 32 * j;
        if (n >= NGPT) continue;
        if (!top && (long long)c2[j] <= fk) continue;   // linked to the layer above: still waiting
        // the run start[j]..k takes this layer's set-1 draw: per 32-layer word,
        // the layers whose threshold it reaches are a prefix of the word's
        // sorted thresholds (RLM:2097-2103)
        const long long v = c1[j];
        for (int w = start[j] >> 5; w <= (k >> 5); ++w) {
          const int lo = max(start[j], 32 * w) - 32 * w, hi = min(k, 32 * w + 31) - 32 * w;
          const uint32_t rm = (hi == 31 ? 0xFFFFFFFFu : ((1u << (hi + 1)) - 1u)) & ~((1u << lo) - 1u);
          const long long* sw = srt + 32 * w;
          int cnt = 0;
#pragma unroll
          for (int st = 16; st >= 1; st >>= 1)
            if (sw[cnt + st - 1] <= v) cnt += st;
          cnt += (sw[31] <= v) ? 1 : 0;   // only when all 32 qualify (then cnt was 31)
          if (w != wi[j]) {
            out[n * nw + wi[j]] = word[j];
            word[j] = 0u;
            wi[j] = w;
          }
          word[j] |= rm & pm[33 * w + cnt];
        }
        start[j] = k + 1;
      }
    } else {
      const long long ak = aux_t[k];
      const long long ck = clr_t[k];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const int n = lane + 32 * j;
        if (n >= NGPT) continue;
        cdf[j] = (k > 0 && (long long)c2[j] < ak) ? cdf[j] : c1[j];
        if ((long long)cdf[j] >= ck) word[j] |= 1u << (k & 31);
        if ((k & 31) == 31 || k == nlay - 1) {
          out[n * nw + (k >> 5)] = word[j];
          word[j] = 0u;
        }
      }
    }
  }
  if (iovr == 3) {
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const int n = lane + 32 * j;
      if (n < NGPT) out[n * nw + wi[j]] = word[j];
    }
  }
}

// The draws of random (iovr=0) and maximum-random (iovr=1) overlap come from
// a ring that holds the raw (untempered) twister sequence itself: sequence
// index s (x_0..x_623 = the seeding, draw p = tempered x_{624+p}) sits at
// ring[s mod cap].  A twist appends the next 624 words in place,
//   x_{j+t} = mt_word(x_{j+t-624}, x_{j+t-623}, x_{j+t-227}),
// so there is no separate state array and no copy; cap is a multiple of
// 624, so neither the block being written nor the one before it wraps.
// Lanes walk g-points in rounds of kMcicaRound (5 x 28 = 140): the ring
// holds one round's draws plus the twist history.
constexpr int kMcicaRound = 28;

__host__ __device__ constexpr uint32_t temper_c(uint32_t y) {
  return ((((y ^ (y >> 11)) ^ (((y ^ (y >> 11)) << 7) & kTmaskB)) ^
           ((((y ^ (y >> 11)) ^ (((y ^ (y >> 11)) << 7) & kTmaskB)) << 15) & kTmaskC)) ^
          (((((y ^ (y >> 11)) ^ (((y ^ (y >> 11)) << 7) & kTmaskB)) ^
             ((((y ^ (y >> 11)) ^ (((y ^ (y >> 11)) << 7) & kTmaskB)) << 15) & kTmaskC)) >>
            18)));
}
static_assert(temper_c(kRawAllOnes) == 0xFFFFFFFFu, "kRawAllOnes tempers to 2^32 - 1");

// Per-warp shared memory: clear[nlay] = 1 - cldf (double), ring[cap].  For
// iovr 3..5 the ring's space holds the two twister states and the per-layer
// overlap parameter instead.
__host__ __device__ inline size_t mcica_warp_bytes(int nlay, int cap) {
  return ((nlay * 8 + 15) & ~15) + (size_t)cap * 4;
}

constexpr int kMcicaWarps = 6;   // 6 warps x 18.5 KB (127 layers): two CTAs, twelve warps per SM

// NG g-points per column: 140 for the longwave path (every overlap, block or
// stage inputs), 112 for the shortwave path (stage inputs, iovr 0..2: the
// shortwave decorrelation-length and exponential overlaps draw in another
// order, radsw_main.F90:2101-2198, and are not built here).
template <int NG>
__global__ void __launch_bounds__(32 * kMcicaWarps)
lw_mcica_kernel(const Block* __restrict__ blocks, int nblocks, const Block b0, int ncols, McicaArgs a,
                uint32_t* __restrict__ bits) {
  extern __shared__ __align__(16) char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const size_t wbytes = mcica_warp_bytes(a.nlay, a.cap);
  char* my = smem_raw + wbytes * wib;
  double* clr = reinterpret_cast<double*>(my);   // 1 - cldf(k), used by every test of the walk
  uint32_t* ring = reinterpret_cast<uint32_t*>(my + ((a.nlay * 8 + 15) & ~15));
  const int nlay = a.nlay, nlp1 = nlay + 1, cap = a.cap;
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
      seed = (a.isubclw == 1) ? 140 + (B.seed0 + i + 1) : B.icseed[i];   // RLM:765-773
    } else {
      for (int k = lane; k < nlay; k += 32) {
        clr[k] = 1.0 - a.st.cldf[c + (size_t)a.st.ld * k];
      }
      any = true;
      seed = a.st.seed[c];
    }
    if (!__any_sync(0xffffffffu, any)) continue;   // clear column: no draws
    const uint32_t s0 = (uint32_t)(seed == 0 ? 4357 : seed);   // random_setseed_t (MT:285-299)

    uint32_t* out = bits + (size_t)c * NG * a.nw;
    if constexpr (NG == NGPT) {
    if (a.iovr >= 3) {
      // two sequence rings, the per-layer overlap parameter and the walk's
      // thresholds in the ring's space
      uint32_t* mtA = ring;
      uint32_t* mtB = ring + kTwoSetRing;
      double* aux = reinterpret_cast<double*>(ring + 2 * kTwoSetRing);
      const Block* B = (nblocks > 0) ? ((nblocks == 1) ? &b0 : &blocks[find_block(blocks, nblocks, c)]) : nullptr;
      const int i = B ? c - B->col0 : 0;
      if (a.iovr == 3) {
        // fac_lcf(k) = exp(-0.5 (dz(k) + dz(k-1)) / de_lgth), dz in the internal order (RLM:819, 2001)
        const double dl = B ? B->in[F_DELGTH][i] : a.st.delg[c];
        for (int k = 1 + lane; k < nlay; k += 32) {
          double dz0, dz1;
          if (B) {
            const int r0 = a.top_at_1 ? nlp1 - (k + 1) - 1 : k, r1 = a.top_at_1 ? nlp1 - k - 1 : k - 1;
            dz0 = B->in[F_DZLYR][i + (size_t)B->ld * r0];
            dz1 = B->in[F_DZLYR][i + (size_t)B->ld * r1];
          } else {
            dz0 = a.st.dz[c + (size_t)a.st.ld * k];
            dz1 = a.st.dz[c + (size_t)a.st.ld * (k - 1)];
          }
          aux[k] = exp(-0.5 * (dz0 + dz1) / dl);
        }
      } else {
        // alpha is taken in the caller's row order, unflipped (RLM:820, 933)
        for (int k = lane; k < nlay; k += 32)
          aux[k] = B ? B->in[F_ALPHA][i + (size_t)B->ld * k] : a.st.alpha[c + (size_t)a.st.ld * k];
      }
      // the walk's integer thresholds, after the rings and aux
      long long* aux_t = reinterpret_cast<long long*>(aux + nlay);
      long long* clr_t = aux_t + nlay;
      __syncwarp();
      for (int k = lane; k < nlay; k += 32) {
        clr_t[k] = umin_ge(clr[k]);
        if (a.iovr == 3) aux_t[k] = (k > 0) ? umax_le(aux[k]) : 0;
        else aux_t[k] = ulim_lt(aux[k]);
      }
      __syncwarp();
      // iovr 3: per 32-layer word, the cloud thresholds in ascending order and,
      // for each count c, the mask of the word's layers with the c smallest
      // (layers past nlay never qualify)
      long long* srt = clr_t + nlay;
      uint32_t* pm = reinterpret_cast<uint32_t*>(srt + 32 * a.nw);
      if (a.iovr == 3) {
        for (int w = 0; w < a.nw; ++w) {
          const int m = 32 * w + lane;
          const long long th = (m < nlay) ? clr_t[m] : LLONG_MAX;
          int rank = 0;
          for (int o = 0; o < 32; ++o) {
            const long long t2 = __shfl_sync(0xffffffffu, th, o);
            rank += (t2 < th || (t2 == th && o < lane)) ? 1 : 0;
          }
          srt[32 * w + rank] = th;
          for (int c = 0; c <= 32; ++c) {
            const uint32_t b = __ballot_sync(0xffffffffu, rank < c);
            if (lane == 0) pm[33 * w + c] = b;
          }
        }
        __syncwarp();
      }
      mcica_two_set(mtA, mtB, clr_t, aux_t, srt, pm, nlay, a.iovr, s0, a.nw, out, lane);
      continue;
    }
    }
    // seeding x_0..x_623 at ring[0..623]: mt(i) = 69069^i seed
    for (int n = lane; n < 624; n += 32) ring[n] = s0 * c_pow69069[n];
    __syncwarp();
    if (a.iovr == 2) {
      // maximum overlap: one draw per g-point, the same at every layer (RLM:1981-1993)
      twist_ring(ring, cap, 624, lane);   // sequence 624..1247 at ring[624..1247] (cap >= 1248)
      for (int n = lane; n < NG; n += 32) {
        double r = u32_unit(temper(ring[624 + n]));
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
    // random (iovr=0) and maximum-random (iovr=1): draw n*nlay+k (RLM:1920-1941)
    long long gen = 624;       // sequence indices generated so far
    int jp = 624;              // gen mod cap
    bool hit = false;          // warp-uniform: some generated word tempers to 2^32 - 1
    static_assert(NG % kMcicaRound == 0, "whole rounds of g-points");
    for (int n0 = 0; n0 < NG; n0 += kMcicaRound) {
      const long long need = 624 + (long long)(n0 + kMcicaRound) * nlay;
      while (gen < need) {
        hit |= __any_sync(0xffffffffu, twist_ring<true>(ring, cap, jp, lane));
        gen += 624;
        jp += 624;
        if (jp == cap) jp = 0;
      }
      const int n = n0 + lane;
      if (!hit) {
        // No draw so far is 1 (only that word tempers to 2^32 - 1), so every
        // cdf stays below 1: a clear layer's flag (cdf >= 1, see below) is 0
        // and the layer after it starts afresh (cdf = r * 1).  Only the
        // cloudy layers are walked, word by word from the warp's mask of them;
        // the flags are those of the walk below, bit for bit.
        const int q0 = (int)((624 + (long long)n * nlay) % cap);
        double cdf = 0.0;
        int kprev = -2;
        for (int w = 0; w < a.nw; ++w) {
          const int kk = 32 * w + lane;
          uint32_t m = __ballot_sync(0xffffffffu, kk < nlay && clr[kk] != 1.0);   // the word's cloudy layers
          if (lane < kMcicaRound) {
            uint32_t word = 0;
            while (m) {
              const int b = __ffs(m) - 1;
              m &= m - 1;
              const int k = 32 * w + b;
              int q = q0 + k;
              if (q >= cap) q -= cap;
              const double r = u32_unit(temper(ring[q]));
              if (k == 0 || a.iovr == 0 || kprev != k - 1) {
                cdf = r;
              } else {
                const double tem1 = clr[k - 1];        // max-random walk (RLM:1949-1960)
                cdf = (cdf > tem1) ? cdf : r * tem1;
              }
              if (cdf >= clr[k]) word |= 1u << b;      // RLM:2097-2103
              kprev = k;
            }
            out[n * a.nw + w] = word;
          }
        }
        __syncwarp();
        continue;
      }
      if (lane < kMcicaRound) {
        int q = (int)((624 + (long long)n * nlay) % cap);
        double cdf = 0.0;
        uint32_t word = 0;
#pragma unroll 4   // lets the ring and cloud-fraction loads of four layers issue ahead
        for (int k = 0; k < nlay; ++k) {
          const uint32_t raw = ring[q];
          if (++q == cap) q = 0;
          const double ck = clr[k];
          if (ck == 1.0) {
            // Clear layer (the same for every lane: lanes are g-points of one layer).
            // Its flag is cdf >= 1, and every draw is <= 1 with equality only for
            // the word that tempers to 2^32 - 1, so the flag needs neither tempering
            // nor conversion: a fresh draw is 1 only for that word, an inherited cdf
            // only if it is 1, and r * tem1 < 1 when tem1 < 1.  The cdf of a clear
            // layer is never read again: the next layer compares it with
            // 1 - cldf = 1 and takes r * 1 = r instead.
            bool bit;
            if (k == 0 || a.iovr == 0) {
              bit = (raw == kRawAllOnes);
            } else {
              const double tem1 = clr[k - 1];
              bit = (tem1 == 1.0) ? (raw == kRawAllOnes) : (cdf > tem1 && cdf >= 1.0);
            }
            if (bit) word |= 1u << (k & 31);
          } else {
            const double r = u32_unit(temper(raw));
            if (k == 0 || a.iovr == 0) {
              cdf = r;
            } else {
              const double tem1 = clr[k - 1];        // max-random walk (RLM:1949-1960)
              cdf = (cdf > tem1) ? cdf : r * tem1;
            }
            if (cdf >= ck) word |= 1u << (k & 31);   // RLM:2097-2103
          }
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

// The raw (untempered) words of one twister stream after
// random_setseed_t(seed) (MT:285-299): out[j] is the state word that draw j
// of random_number_t (MT:330-372) tempers.  One CTA walks the stream; the
// 624-word state is double-buffered in shared memory, so a twist is its
// three dependency phases (words 0..226 from the old state, 227..453 and
// 454..622 from words 227 back in the new one, word 623 from new words 0 and
// 396) with one barrier each and no read-before-write hazard.  Only integer
// work sits on this serial path; tempering and the conversion to a random
// index run later, in parallel, for the words that are used
// (seed_index_of).
constexpr int kSeedThreads = 256;

__global__ void __launch_bounds__(kSeedThreads) lw_seed_stream_kernel(uint32_t seed, long long m,
                                                                      uint32_t* __restrict__ out) {
  __shared__ uint32_t s[2][624];
  const int t = threadIdx.x;
  if (t == 0) {   // MT:290-296, signed wrap = unsigned multiply
    uint32_t v = seed;
    s[0][0] = v;
    for (int i = 1; i < 624; ++i) { v *= 69069u; s[0][i] = v; }
  }
  __syncthreads();
  int cur = 0;
  for (long long base = 0; base < m; base += 624) {
    const uint32_t* o = s[cur];
    uint32_t* w = s[cur ^ 1];
    const long long left = m - base;
    if (t < 227) {   // words 0..226
      const uint32_t v = mt_word(o[t], o[t + 1], o[t + 397]);
      w[t] = v;
      if (t < left) out[base + t] = v;
    }
    __syncthreads();
    if (t < 227) {   // words 227..453
      const int kk = 227 + t;
      const uint32_t v = mt_word(o[kk], o[kk + 1], w[kk - 227]);
      w[kk] = v;
      if (kk < left) out[base + kk] = v;
    }
    __syncthreads();
    if (t < 169) {   // words 454..622
      const int kk = 454 + t;
      const uint32_t v = mt_word(o[kk], o[kk + 1], w[kk - 227]);
      w[kk] = v;
      if (kk < left) out[base + kk] = v;
    } else if (t == 169) {   // word 623
      const uint32_t v = mt_word(o[623], w[0], w[396]);
      w[623] = v;
      if (623 < left) out[base + 623] = v;
    }
    __syncthreads();
    cur ^= 1;
  }
}

// random_index_t (MT:489-503) of one raw word: max(ceiling(h * imax), 1)
// with h = random_number_t's harvest of that word; h * imax rounds as in the
// Fortran (FP64 product, no contraction).
__device__ __forceinline__ int32_t seed_index_of(uint32_t raw, int32_t imax) {
  const double c = ceil(__dmul_rn(u32_unit(temper(raw)), (double)imax));
  return c < 1.0 ? 1 : (int32_t)c;
}

// icsdsw/icsdlw of column ix (GFS_rad_time_vary.fv3.F90:76-82): with
// p = i+isc-1 + (j+jsc-2) cnx (1-based), numrdm(p) and numrdm(p + cnx cny),
// numrdm = random_index(imax) of the face's stream.  A p outside the face
// records the smallest such column in *bad and writes nothing for it.
__global__ void lw_seed_gather_kernel(const uint32_t* __restrict__ raw, const int32_t* __restrict__ imap,
                                      const int32_t* __restrict__ jmap, int n, int isc, int jsc, int cnx,
                                      long long face, int32_t imax, int32_t* icsdsw, int32_t* icsdlw, int* bad) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= n) return;
  const long long p = (long long)imap[ix] + isc - 1 + ((long long)jmap[ix] + jsc - 2) * cnx;
  if (p < 1 || p > face) {
    atomicMin(bad, ix);
    return;
  }
  icsdsw[ix] = seed_index_of(raw[p - 1], imax);
  icsdlw[ix] = seed_index_of(raw[p - 1 + face], imax);
}

// host side ------------------------------------------------------------------

cudaError_t seed_stream_launch(int32_t seed, long long m, uint32_t* raw, cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  const uint32_t s = (uint32_t)(seed == 0 ? 4357 : seed);   // MT:291
  lw_seed_stream_kernel<<<1, kSeedThreads, 0, st>>>(s, m, raw);
  return cudaGetLastError();
}

cudaError_t seed_gather_launch(const uint32_t* raw, const int32_t* imap, const int32_t* jmap, int n, int isc,
                               int jsc, int cnx, long long face, int32_t imax, int32_t* icsdsw, int32_t* icsdlw,
                               int* bad, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  lw_seed_gather_kernel<<<(n + 255) / 256, 256, 0, st>>>(raw, imap, jmap, n, isc, jsc, cnx, face, imax, icsdsw,
                                                         icsdlw, bad);
  return cudaGetLastError();
}

// ring words: one round's draws plus a twist block, and at least the two
// rings, the overlap parameter, the two threshold arrays and the per-word
// sorted thresholds and masks of iovr 3..5; a multiple of 624
int mcica_ring_capacity(int nlay) {
  const long round = (long)kMcicaRound * nlay + 623;
  const long nw = (nlay + 31) / 32;
  const long two_set = 2L * kTwoSetRing + 6L * nlay + 97L * nw;   // + sorted thresholds, prefix masks
  const long need = round > two_set ? round : two_set;
  return (int)((need + 623) / 624 * 624);
}

cudaError_t mcica_prepare(int max_smem) {
  cudaError_t e = cudaFuncSetAttribute(lw_mcica_kernel<NGPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(lw_mcica_kernel<kSwNgpt>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
}

cudaError_t mcica_upload_powers() {
  static uint32_t pw[624];
  pw[0] = 1u;
  for (int i = 1; i < 624; ++i) pw[i] = pw[i - 1] * 69069u;
  return cudaMemcpyToSymbol(c_pow69069, pw, sizeof(pw));
}

cudaError_t mcica_launch(const Block* blocks, int nblocks, const Block& b0, int ncols, int nlay, int iovr, int isubclw,
                         int top_at_1, const McicaStage& stage, uint32_t* bits, int num_sms, cudaStream_t st) {
  McicaArgs a;
  a.nlay = nlay;
  a.nw = (nlay + 31) / 32;
  a.iovr = iovr;
  a.isubclw = isubclw;
  a.top_at_1 = top_at_1;
  a.cap = mcica_ring_capacity(nlay);
  a.st = stage;
  const int wpb = kMcicaWarps;
  size_t smem = mcica_warp_bytes(nlay, a.cap) * wpb;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lw_mcica_kernel<NGPT>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  int grid = min((ncols + wpb - 1) / wpb, num_sms * per_sm);
  if (grid < 1) return cudaSuccess;
  lw_mcica_kernel<NGPT><<<grid, wpb * 32, smem, st>>>(blocks, nblocks, b0, ncols, a, bits);
#if LW_DEBUG_CHECKS
  {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { fprintf(stderr, "lw debug: mcica kernel failed\n"); return e; }
  }
#endif
  return cudaGetLastError();
}

// Shortwave sub-columns with decorrelation-length (iovr 3) or exponential /
// exponential-random (iovr 4, 5) overlap (radsw_main.F90:2101-2198).  Both
// random sets are g-major, set 1 = draws [0, 112 nlay) and set 2 = draws
// [112 nlay, 224 nlay) of one stream, cdfunc(k, n) = draw (n-1) nlay + k.
// Set 2 is read from a second sequence ring that runs 112 nlay draws ahead
// of the first; each ring holds one round's draws plus the twist history,
// as in the iovr 0/1 walk.  Each lane walks its g-point: top-down for iovr
// 3 (cdfunc(k) = cdfunc(k+1) when cdfun2(k) <= fac_lcf(k+1)), bottom-up for
// 4, 5 (cdfunc(k) = cdfunc(k-1) when cdfun2(k) < alpha(k)), flagging
// cdfunc(k) >= 1 - cldf(k).  stage.alpha holds fac_lcf (iovr 3, entry k is
// the factor between layers k-1 and k) or alpha (iovr 4, 5), per layer in
// internal order.
constexpr int kSwTwoSetMaxWarps = 8;   // warps per CTA: as many as the shared memory holds, up to 8

__host__ __device__ inline size_t sw_two_set_warp_bytes(int nlay, int cap) {
  return 2 * (((size_t)nlay * 8 + 15) & ~(size_t)15) + 2 * (size_t)cap * 4;
}

__global__ void __launch_bounds__(32 * kSwTwoSetMaxWarps)
sw_mcica_two_set_kernel(int ncols, McicaArgs a, uint32_t* __restrict__ bits) {
  extern __shared__ __align__(16) char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nlay = a.nlay, cap = a.cap, nw = a.nw;
  const size_t lb = ((size_t)nlay * 8 + 15) & ~(size_t)15;
  char* my = smem_raw + sw_two_set_warp_bytes(nlay, cap) * wib;
  double* clr = reinterpret_cast<double*>(my);         // 1 - cldf(k)
  double* aux = reinterpret_cast<double*>(my + lb);    // fac_lcf or alpha
  uint32_t* ra = reinterpret_cast<uint32_t*>(my + 2 * lb);
  uint32_t* rb = ra + cap;
  const int wpb = blockDim.x >> 5;
  const int warps_total = gridDim.x * wpb;
  const long long P0 = (long long)kSwNgpt * nlay;   // set 2 starts here
  for (int c = blockIdx.x * wpb + wib; c < ncols; c += warps_total) {
    __syncwarp();
    for (int k = lane; k < nlay; k += 32) {
      clr[k] = 1.0 - a.st.cldf[c + (size_t)a.st.ld * k];
      aux[k] = a.st.alpha[c + (size_t)a.st.ld * k];
    }
    const int32_t seed = a.st.seed[c];
    const uint32_t s0 = (uint32_t)(seed == 0 ? 4357 : seed);   // random_setseed_t (MT:285-299)
    for (int n = lane; n < 624; n += 32) ra[n] = rb[n] = s0 * c_pow69069[n];
    __syncwarp();
    long long ga = 624, gb = 624;    // sequence words generated in each ring
    int ja = 624 % cap, jb = 624 % cap;
    uint32_t* out = bits + (size_t)c * kSwNgpt * nw;
    for (int n0 = 0; n0 < kSwNgpt; n0 += kMcicaRound) {
      const long long need_a = 624 + (long long)(n0 + kMcicaRound) * nlay;
      while (ga < need_a) {
        twist_ring(ra, cap, ja, lane);
        ga += 624;
        ja += 624;
        if (ja == cap) ja = 0;
      }
      const long long need_b = need_a + P0;
      while (gb < need_b) {
        twist_ring(rb, cap, jb, lane);
        gb += 624;
        jb += 624;
        if (jb == cap) jb = 0;
      }
      const int n = n0 + lane;
      if (lane < kMcicaRound) {
        const int qa = (int)((624 + (long long)n * nlay) % cap);
        const int qb = (int)((624 + P0 + (long long)n * nlay) % cap);
        auto at = [&](const uint32_t* r, int q0, int k) {
          int q = q0 + k;
          if (q >= cap) q -= cap;
          return u32_unit(temper(r[q]));
        };
        uint32_t word = 0;
        if (a.iovr == 3) {
          double cur = at(ra, qa, nlay - 1);
          for (int k = nlay - 1; k >= 0; --k) {
            if (k < nlay - 1 && !(at(rb, qb, k) <= aux[k + 1])) cur = at(ra, qa, k);
            if (cur >= clr[k]) word |= 1u << (k & 31);
            if ((k & 31) == 0) {
              out[n * nw + (k >> 5)] = word;
              word = 0;
            }
          }
        } else {
          double cur = 0.0;
          for (int k = 0; k < nlay; ++k) {
            if (k == 0 || !(at(rb, qb, k) < aux[k])) cur = at(ra, qa, k);
            if (cur >= clr[k]) word |= 1u << (k & 31);
            if ((k & 31) == 31 || k == nlay - 1) {
              out[n * nw + (k >> 5)] = word;
              word = 0;
            }
          }
        }
      }
      __syncwarp();
    }
  }
}

cudaError_t mcica_sw_two_set_prepare(int max_smem) {
  return cudaFuncSetAttribute(sw_mcica_two_set_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
}

cudaError_t mcica_sw_two_set_launch(int ncols, int nlay, int iovr, const McicaStage& stage, uint32_t* bits,
                                    int num_sms, cudaStream_t st) {
  if (iovr < 3 || iovr > 5) return cudaErrorInvalidValue;
  McicaArgs a;
  a.nlay = nlay;
  a.nw = (nlay + 31) / 32;
  a.iovr = iovr;
  a.isubclw = 2;
  a.top_at_1 = 0;
  const long round = (long)kMcicaRound * nlay + 623;
  a.cap = (int)((round + 623) / 624 * 624);
  a.st = stage;
  static const int max_smem = [] {   // initialised once, thread-safe
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
  }();
  const size_t per_warp = sw_two_set_warp_bytes(nlay, a.cap);
  const int wpb = (int)std::min<size_t>(kSwTwoSetMaxWarps, (size_t)max_smem / per_warp);
  if (wpb < 1) return cudaErrorInvalidValue;
  const size_t smem = per_warp * wpb;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sw_mcica_two_set_kernel, 32 * wpb, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = min((ncols + wpb - 1) / wpb, num_sms * per_sm);
  if (grid < 1) return cudaSuccess;
  sw_mcica_two_set_kernel<<<grid, 32 * wpb, smem, st>>>(ncols, a, bits);
  return cudaGetLastError();
}

// Shortwave sub-columns (mcica_subcol, radsw_main.F90:1952-2212) for iovr 0
// (random), 1 (maximum-random) and 2 (maximum): the draws are g-major,
// rand2d((n-1)*nlay + k) as in the longwave generator, over 112 g-points.
// stage.cldf is the layer cloud fraction floored at ftiny = 1e-12
// (radsw_main.F90:1904-1908), internal (surface-first) order.
cudaError_t mcica_sw_launch(int ncols, int nlay, int iovr, const McicaStage& stage, uint32_t* bits, int num_sms,
                            cudaStream_t st) {
  if (iovr < 0 || iovr > 2) return cudaErrorInvalidValue;
  McicaArgs a;
  a.nlay = nlay;
  a.nw = (nlay + 31) / 32;
  a.iovr = iovr;
  a.isubclw = 2;
  a.top_at_1 = 0;
  a.cap = mcica_ring_capacity(nlay);
  a.st = stage;
  const int wpb = kMcicaWarps;
  size_t smem = mcica_warp_bytes(nlay, a.cap) * wpb;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lw_mcica_kernel<kSwNgpt>, wpb * 32, smem);
  if (per_sm < 1) per_sm = 1;
  int grid = min((ncols + wpb - 1) / wpb, num_sms * per_sm);
  if (grid < 1) return cudaSuccess;
  Block none{};
  lw_mcica_kernel<kSwNgpt><<<grid, wpb * 32, smem, st>>>(nullptr, 0, none, ncols, a, bits);
  return cudaGetLastError();
}

}  // namespace lw
