// smc_common.cuh -- shared device code of libvsmc_cuda (sm_100a only).
//
// Counter-based RNG in registers, the libstdc++-compatible uniform and polar
// normal transforms, block reductions and the deterministic tile "spine".
// All double arithmetic that has to reproduce the reference's rounding is
// written with explicit __dadd_rn/__dmul_rn/__ddiv_rn so that nvcc cannot
// contract it into FMAs.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/vsmc_cuda.h"

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
        x = __dadd_rn(__dmul_rn(2.0, canonical_u32x2(w.x, w.y)), -1.0);
        y = __dadd_rn(__dmul_rn(2.0, canonical_u32x2(w.z, w.w)), -1.0);
        r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    } while (r2 > 1.0 || r2 == 0.0);
}

// Exact polar point of one Philox block (two canonical doubles).
__device__ __forceinline__ void polar_point(const uint4 &w, double &x,
                                            double &y, double &r2)
{
    x = __dadd_rn(__dmul_rn(2.0, canonical_u32x2(w.x, w.y)), -1.0);
    y = __dadd_rn(__dmul_rn(2.0, canonical_u32x2(w.z, w.w)), -1.0);
    r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

__device__ __forceinline__ bool polar_ok(double r2)
{
    return !(r2 > 1.0 || r2 == 0.0);
}

// The first two accepted polar points of a particle stream (libstdc++'s
// two calls of the polar loop).  Three blocks are drawn up front: their
// Philox chains are independent, so they overlap in the pipeline, and 88%
// of particles need no more; the rest continue one block at a time.  The
// points are exactly those of the sequential loop, in stream order.
__device__ __forceinline__ void polar_two(uint32_t iter, uint32_t id,
                                          uint32_t stream, uint32_t k0,
                                          uint32_t k1, double &x1, double &y1,
                                          double &q1, double &x2, double &y2,
                                          double &q2)
{
    uint4 w[3];
    double x[3], y[3], r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        w[k] = philox4x32_10(make_uint4((uint32_t)(k + 1), iter, id, stream),
                             k0, k1);
        polar_point(w[k], x[k], y[k], r[k]);
    }
    int n = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (polar_ok(r[k])) {
            if (n == 0) {
                x1 = x[k];
                y1 = y[k];
                q1 = r[k];
            } else if (n == 1) {
                x2 = x[k];
                y2 = y[k];
                q2 = r[k];
            }
            ++n;
        }
    }
    if (n < 2) {
        PhiloxStream s;
        s.ctr = make_uint4(3u, iter, id, stream);
        s.k0 = k0;
        s.k1 = k1;
        double a, b, c;
        while (n < 2) {
            polar_point(s.next_block(), a, b, c);
            if (polar_ok(c)) {
                if (n == 0) {
                    x1 = a;
                    y1 = b;
                    q1 = c;
                } else {
                    x2 = a;
                    y2 = b;
                    q2 = c;
                }
                ++n;
            }
        }
    }
}

// mult = sqrt(-2 log(r2) / r2); the distribution returns y*mult first and
// caches x*mult.
__device__ __forceinline__ double polar_mult_f64(double r2)
{
    return __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
}

__device__ __forceinline__ float polar_mult_f32(double r2)
{
    const float r2f = static_cast<float>(r2);
    return sqrtf(-2.0f * logf(r2f) / r2f);
}

// --------------------------------------------------------- reductions ------
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ long long warp_sum_ll(long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Inclusive warp scan (Hillis-Steele over shuffles).
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o)
            v += n;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total.  `sh` needs blockDim.x/32 entries.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *sh, T &total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    const T inc = warp_incl_scan(v);
    if (lane == 31)
        sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T s = lane < nw ? sh[lane] : T(0);
        s = warp_incl_scan(s);
        if (lane < nw)
            sh[lane] = s;
    }
    __syncthreads();
    const T wexcl = wid > 0 ? sh[wid - 1] : T(0);
    total = sh[nw - 1];
    __syncthreads();
    return wexcl + inc - v;
}

// Online log-sum-exp accumulator: m = running max, s1 = sum exp(lw - m),
// s2 = sum exp(2 (lw - m)), sx/sy = sum exp(lw - m) * (x, y).
struct LseAcc {
    double m, s1, s2, sx, sy;

    __device__ __forceinline__ void init()
    {
        m = -INFINITY;
        s1 = s2 = sx = sy = 0.0;
    }

    __device__ __forceinline__ void rescale_to(double nm)
    {
        if (nm == m)
            return;
        const double f = (m == -INFINITY) ? 0.0 : exp(m - nm);
        s1 *= f;
        s2 *= f * f;
        sx *= f;
        sy *= f;
        m = nm;
    }

    __device__ __forceinline__ void add(double lw, double x, double y)
    {
        if (!(lw <= m)) { // new max (or NaN: propagate below)
            if (lw != lw) {
                s1 = lw;
                return;
            }
            rescale_to(lw);
        }
        if (lw == -INFINITY)
            return;
        const double e = exp(lw - m);
        s1 += e;
        s2 += e * e;
        sx += e * x;
        sy += e * y;
    }

    __device__ __forceinline__ void merge(const LseAcc &o)
    {
        if (o.m == -INFINITY && o.s1 == 0.0)
            return;
        const double nm = fmax(m, o.m);
        const double fa = (m == -INFINITY) ? 0.0 : exp(m - nm);
        const double fb = (o.m == -INFINITY) ? 0.0 : exp(o.m - nm);
        s1 = s1 * fa + o.s1 * fb;
        s2 = s2 * fa * fa + o.s2 * fb * fb;
        sx = sx * fa + o.sx * fb;
        sy = sy * fa + o.sy * fb;
        m = nm;
    }
};

__device__ __forceinline__ LseAcc shfl_xor(const LseAcc &a, int o)
{
    LseAcc b;
    b.m = __shfl_xor_sync(0xffffffffu, a.m, o);
    b.s1 = __shfl_xor_sync(0xffffffffu, a.s1, o);
    b.s2 = __shfl_xor_sync(0xffffffffu, a.s2, o);
    b.sx = __shfl_xor_sync(0xffffffffu, a.sx, o);
    b.sy = __shfl_xor_sync(0xffffffffu, a.sy, o);
    return b;
}

// Deterministic block reduction of LseAcc (fixed shuffle tree, fixed warp
// order), result valid in thread 0.
__device__ __forceinline__ LseAcc block_reduce_lse(LseAcc a, LseAcc *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        a.merge(shfl_xor(a, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
        sh[wid] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        LseAcc r = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            r.merge(sh[w]);
        sh[0] = r;
    }
    __syncthreads();
    LseAcc r = sh[0];
    __syncthreads();
    return r;
}

} // namespace vsmc_b200
