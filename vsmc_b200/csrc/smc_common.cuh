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
#include "../../include/vsmc_b200/smc_device.cuh"

namespace vsmc_b200 {

// Philox blocks a particle draws up front for its two polar points.  Four
// measured best at 2^24 particles (the FP64 move 0.692 ms with three, 0.684
// with four, 0.70 with five and 0.73 with six, which spill).
#ifndef VSMC_POLAR_UPFRONT
#define VSMC_POLAR_UPFRONT 4
#endif

// The first two accepted polar points of a particle stream (libstdc++'s
// two calls of the polar loop).  VSMC_POLAR_UPFRONT blocks are drawn up
// front: their Philox chains are independent, so they overlap in the
// pipeline, and with four 97% of particles need no more (88% with three,
// and a warp with any such lane runs the extra block anyway); the rest
// continue one block at a time.  The points are exactly those of the
// sequential loop, in stream order.
__device__ __forceinline__ void polar_two(uint32_t iter, uint32_t id,
                                          uint32_t stream, uint32_t k0,
                                          uint32_t k1, double &x1, double &y1,
                                          double &q1, double &x2, double &y2,
                                          double &q2)
{
    constexpr int U = VSMC_POLAR_UPFRONT;
    uint4 w[U];
    double x[U], y[U], r[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
        w[k] = philox4x32_10(make_uint4((uint32_t)(k + 1), iter, id, stream),
                             k0, k1);
        polar_point(w[k], x[k], y[k], r[k]);
    }
    int n = 0;
#pragma unroll
    for (int k = 0; k < U; ++k) {
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
        s.ctr = make_uint4((uint32_t)U, iter, id, stream);
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
    return __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, fm::fm_log(r2)), r2));
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
