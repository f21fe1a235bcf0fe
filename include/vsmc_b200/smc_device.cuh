// smc_device.cuh -- device building blocks shared by libvsmc_cuda and by
// programs that compile their own particle moves against it (nvcc, sm_100a).
//
// * Philox4x32-10 and Threefry4x64-20 blocks in registers and the counter
//   arithmetic of vSMC's engines (include/vsmc/rng/philox.hpp,
//   threefry.hpp, utility/counter.hpp);
// * libstdc++'s uniform conversions (generate_canonical) and the polar
//   method's attempt of std::normal_distribution;
// * the per-tile weight statistics a move writes and the library's
//   normalisation / ESS / resampling kernels read (TileStats, with the
//   online log-sum-exp accumulator that fills it).
//
// All double arithmetic that has to reproduce the reference's rounding is
// written with explicit __dadd_rn/__dmul_rn/__ddiv_rn so that nvcc cannot
// contract it into FMAs.
#ifndef VSMC_B200_SMC_DEVICE_CUH
#define VSMC_B200_SMC_DEVICE_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "fastmath.cuh"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ != 1000)
#error "libvsmc_cuda is written for sm_100a (B200) only"
#endif

namespace vsmc_b200 {

constexpr int kThreads = 256;           // threads per CTA on streaming kernels
constexpr int kItems = 8;               // particles per thread per tile
constexpr int kTile = kThreads * kItems; // particles per tile (2048)
constexpr int kSpineThreads = 1024;     // one CTA scans the per-tile spine

// ------------------------------------------------------------ Philox ------
// Philox4x32-10 (vSMC include/vsmc/rng/philox.hpp:137-265, 504-523): key
// bumped by the Weyl constants before rounds 2..10; round =
// (hi(M1*s2)^k0^s1, lo(M1*s2), hi(M0*s0)^k1^s3, lo(M0*s0)).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0,
                                               uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        // one 32x32->64 wide multiply gives both halves of each product
        const unsigned long long pa = (unsigned long long)0xCD9E8D57u * c.z;
        const unsigned long long pb = (unsigned long long)0xD2511F53u * c.x;
        c = make_uint4((uint32_t)(pa >> 32) ^ k0 ^ c.y, (uint32_t)pa,
                       (uint32_t)(pb >> 32) ^ k1 ^ c.w, (uint32_t)pb);
    }
    return c;
}

// ---------------------------------------------------------- Threefry ------
struct u64x4 {
    uint64_t v[4];
};

__device__ __forceinline__ uint64_t rotl64(uint64_t x, unsigned r)
{
    return (x << r) | (x >> (64 - r));
}

// Threefry4x64-20 (vSMC include/vsmc/rng/threefry.hpp:105-233, 473-506):
// Threefish-256 rotations, key injection every 4 rounds with the parity word
// 0x1BD11BDAA9FC1A22 ^ k0 ^ k1 ^ k2 ^ k3.
__device__ __forceinline__ u64x4 threefry4x64_20(u64x4 c, const u64x4 &k)
{
    uint64_t p[5];
    p[4] = 0x1BD11BDAA9FC1A22ull;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        p[i] = k.v[i];
        p[4] ^= k.v[i];
    }
    constexpr unsigned R0[8] = {14, 52, 23, 5, 25, 46, 58, 32};
    constexpr unsigned R1[8] = {16, 57, 40, 37, 33, 12, 22, 32};
    uint64_t b0 = c.v[0] + p[0], b1 = c.v[1] + p[1], b2 = c.v[2] + p[2],
             b3 = c.v[3] + p[3];
#pragma unroll
    for (unsigned n = 1; n <= 20; ++n) {
        const unsigned r = (n - 1) % 8;
        if (n % 2) { // pairs (0,1) and (2,3)
            b0 += b1;
            b1 = rotl64(b1, R0[r]) ^ b0;
            b2 += b3;
            b3 = rotl64(b3, R1[r]) ^ b2;
        } else { // pairs (0,3) and (2,1)
            b0 += b3;
            b3 = rotl64(b3, R0[r]) ^ b0;
            b2 += b1;
            b1 = rotl64(b1, R1[r]) ^ b2;
        }
        if (n % 4 == 0) {
            const unsigned s = n / 4;
            b0 += p[(s + 0) % 5];
            b1 += p[(s + 1) % 5];
            b2 += p[(s + 2) % 5];
            b3 += p[(s + 3) % 5] + s;
        }
    }
    u64x4 o;
    o.v[0] = b0;
    o.v[1] = b1;
    o.v[2] = b2;
    o.v[3] = b3;
    return o;
}

// Block number `blk` (>= 1) after base counter c0 for a 4x64 engine:
// little-endian add with carry (utility/counter.hpp:180-192).
__device__ __forceinline__ u64x4 ctr64_add(const u64x4 &c0, uint64_t blk)
{
    u64x4 c = c0;
    uint64_t carry = blk;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint64_t s = c.v[i] + carry;
        carry = (s < c.v[i]) ? 1 : 0;
        c.v[i] = s;
    }
    return c;
}

// Word at stream offset w (0-based) of a Threefry4x64 engine whose next word
// is lane 0 of block c0 + 1.
__device__ __forceinline__ uint64_t threefry_word(const u64x4 &key,
                                                  const u64x4 &c0, uint64_t w)
{
    const u64x4 b = threefry4x64_20(ctr64_add(c0, w / 4 + 1), key);
    return b.v[w % 4];
}

// ---------------------------------------------------- uniform transforms --
// libstdc++ generate_canonical<double,53> over a 64-bit engine: one word,
// double(x) * 2^-64, a rounded-up 1.0 replaced by the largest double < 1.
__device__ __forceinline__ double canonical_u64(uint64_t x)
{
    const double r = __dmul_rn(__ull2double_rn(x), 0x1p-64);
    return r >= 1.0 ? 0x1.fffffffffffffp-1 : r;
}

// ... over a 32-bit engine: two words, (a + b * 2^32) * 2^-64 with a single
// rounding of the sum.
// The exact sum a + b*2^32 is the 64-bit integer (b << 32) | a, so its one
// rounding to double is a single 64-bit conversion.
__device__ __forceinline__ double canonical_u32x2(uint32_t a, uint32_t b)
{
    const unsigned long long x = ((unsigned long long)b << 32) | a;
    const double r = __dmul_rn(__ull2double_rn(x), 0x1p-64);
    return r >= 1.0 ? 0x1.fffffffffffffp-1 : r;
}

// 2U - 1 of the canonical double U above, in one rounding: with d the
// rounded 64-bit integer, 2U = d * 2^-63 is exact, so fma(d, 2^-63, -1)
// rounds d * 2^-63 - 1 once, exactly as 2U - 1 does.  When d rounds up to
// 2^64, U is clamped to 1 - 2^-53 and 2U - 1 is 1 - 2^-52; the fma gives 1.0
// there and is clamped to the same value.
__device__ __forceinline__ double polar_coord_u32x2(uint32_t a, uint32_t b)
{
    const unsigned long long x = ((unsigned long long)b << 32) | a;
    const double r = __fma_rn(__ull2double_rn(x), 0x1p-63, -1.0);
    return r >= 1.0 ? 0x1.ffffffffffffep-1 : r;
}

// ------------------------------------------------------ polar normals ------
// A Philox4x32 stream positioned at a block boundary: every polar attempt of
// libstdc++'s normal_distribution consumes exactly four 32-bit words (two
// canonical doubles), i.e. one Philox block.  The stream state is therefore
// just the next block counter.
struct PhiloxStream {
    uint4 ctr; // counter of the NEXT block minus one (increment-before-use)
    uint32_t k0, k1;

    __device__ __forceinline__ uint4 next_block()
    {
        // Counter<Array<uint32_t,4>>::increment: carry from word 0.
        if (++ctr.x == 0)
            if (++ctr.y == 0)
                if (++ctr.z == 0)
                    ++ctr.w;
        return philox4x32_10(ctr, k0, k1);
    }
};

// One accepted point of libstdc++'s polar method (normal_distribution::
// operator()): x, y = 2U - 1 from two canonical draws; reject r2 > 1 or
// r2 == 0.  The acceptance test is exact double arithmetic on the same words
// in both precision forms, so every form consumes the stream identically.
__device__ __forceinline__ void polar_accept(PhiloxStream &s, double &x,
                                             double &y, double &r2)
{
    do {
        const uint4 w = s.next_block();
        x = polar_coord_u32x2(w.x, w.y);
        y = polar_coord_u32x2(w.z, w.w);
        r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    } while (r2 > 1.0 || r2 == 0.0);
}

// Exact polar point of one Philox block (two canonical doubles).
__device__ __forceinline__ void polar_point(const uint4 &w, double &x,
                                            double &y, double &r2)
{
    x = polar_coord_u32x2(w.x, w.y);
    y = polar_coord_u32x2(w.z, w.w);
    r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

__device__ __forceinline__ bool polar_ok(double r2)
{
    return !(r2 > 1.0 || r2 == 0.0);
}

// Per-tile statistics of the new log-weights: online log-sum-exp (m, s1, s2),
// the weighted position sums (sx, sy) and the sums of the gathered previous
// positions (gx, gy) for the monitor of a resampled step.
struct TileStats {
    double m, s1, s2, sx, sy, gx, gy, pad;
};

__device__ __forceinline__ double lse_exp(double v) { return fm::fm_exp(v); }
__device__ __forceinline__ double lse_exp(float v) { return (double)expf(v); }

// Per-thread weight statistics against a lazy reference: the first finite
// log-weight becomes the reference and later values are accumulated as
// exp(lw - ref) even above it (double has the range), so the exponential is
// evaluated once per particle; the reference moves only when a value
// exceeds it by more than kLazy (then exp^2 could overflow).  mx tracks the
// true maximum.
struct LseRef {
    double ref, mx, s1, s2, sx, sy;

    __device__ __forceinline__ void init()
    {
        ref = -INFINITY;
        mx = -INFINITY;
        s1 = s2 = sx = sy = 0.0;
    }
};

template <typename Real>
struct LazyBound;
template <>
struct LazyBound<double> {
    static constexpr double v = 300.0;
};
template <>
struct LazyBound<float> {
    static constexpr double v = 40.0;
};

template <typename Real>
__device__ __forceinline__ void lse_add(LseRef &a, Real lw, Real x, Real y)
{
    const double l = (double)lw;
    if (l != l) {
        a.s1 = l; // NaN propagates to the degenerate check
        return;
    }
    if (l == -INFINITY)
        return;
    a.mx = fmax(a.mx, l);
    if (a.ref == -INFINITY) {
        a.ref = l;
    } else if (l - a.ref > LazyBound<Real>::v) {
        const double f = fm::fm_exp(a.ref - l);
        a.s1 *= f;
        a.s2 *= f * f;
        a.sx *= f;
        a.sy *= f;
        a.ref = l;
    }
    const double e = lse_exp((Real)(lw - (Real)a.ref));
    a.s1 += e;
    a.s2 += e * e;
    a.sx += e * (double)x;
    a.sy += e * (double)y;
}

// Rescale a thread's sums to the common maximum M: exp(ref - M) <= 1.
__device__ __forceinline__ void lse_rescale(LseRef &a, double M)
{
    const double f = a.ref == -INFINITY ? 0.0 : fm::fm_exp(a.ref - M);
    a.s1 *= f;
    a.s2 *= f * f;
    a.sx *= f;
    a.sy *= f;
    a.ref = M;
}

__device__ __forceinline__ double warp_max_nan(double v, unsigned width)
{
    for (unsigned o = width / 2; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum of the rescaled statistics over `width` lanes.
__device__ __forceinline__ void warp_sum_stats(LseRef &a, double &gx,
                                               double &gy, unsigned width)
{
    for (unsigned o = width / 2; o > 0; o >>= 1) {
        a.s1 += __shfl_xor_sync(0xffffffffu, a.s1, o);
        a.s2 += __shfl_xor_sync(0xffffffffu, a.s2, o);
        a.sx += __shfl_xor_sync(0xffffffffu, a.sx, o);
        a.sy += __shfl_xor_sync(0xffffffffu, a.sy, o);
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
        gy += __shfl_xor_sync(0xffffffffu, gy, o);
    }
}


// The tile's statistics from every thread's accumulator (acc, plus the sums
// gx, gy of gathered positions, 0 where unused): per warp a common maximum,
// one rescale per lane and plain sums in a fixed shuffle tree; then warp 0
// joins the NW warps in the same way and writes *out.  `sh_w` holds
// 7 x NW doubles; one barrier (callers that run several tiles alternate two
// such buffers).  Every thread of the CTA calls it.
template <int NW>
__device__ __forceinline__ void tile_stats_reduce(LseRef acc, double gx,
                                                  double gy, double *sh_w,
                                                  TileStats *out)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const double wm = warp_max_nan(acc.mx, 32);
    lse_rescale(acc, wm);
    warp_sum_stats(acc, gx, gy, 32);
    if (lane == 0) {
        double *w = sh_w;
        w[0 * NW + wid] = wm;
        w[1 * NW + wid] = acc.s1;
        w[2 * NW + wid] = acc.s2;
        w[3 * NW + wid] = acc.sx;
        w[4 * NW + wid] = acc.sy;
        w[5 * NW + wid] = gx;
        w[6 * NW + wid] = gy;
    }
    __syncthreads();
    if (wid == 0) {
        const double *w = sh_w;
        LseRef r;
        double tx = 0.0, ty = 0.0;
        r.init();
        if (lane < NW) {
            r.ref = w[0 * NW + lane];
            r.mx = r.ref;
            r.s1 = w[1 * NW + lane];
            r.s2 = w[2 * NW + lane];
            r.sx = w[3 * NW + lane];
            r.sy = w[4 * NW + lane];
            tx = w[5 * NW + lane];
            ty = w[6 * NW + lane];
        }
        const double tm = warp_max_nan(r.mx, NW);
        lse_rescale(r, tm);
        warp_sum_stats(r, tx, ty, NW);
        if (lane == 0) {
            TileStats ts;
            ts.m = tm;
            ts.s1 = r.s1;
            ts.s2 = r.s2;
            ts.sx = r.sx;
            ts.sy = r.sy;
            ts.gx = tx;
            ts.gy = ty;
            ts.pad = 0.0;
            *out = ts;
        }
    }
}

} // namespace vsmc_b200

#endif // VSMC_B200_SMC_DEVICE_CUH
