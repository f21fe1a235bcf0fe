// exact_scan.cuh -- the reference's sequential cumulative weight, exactly,
// computed in parallel.
//
// internal::inversion (resample/common.hpp:76-79) walks the weights with
// `accw += weight[i]`: S_i = fl(S_{i-1} + w_i), S_{-1} = 0, one rounding
// per step.  A parallel scan rounds differently, so a uniform lying within
// the scan's error of a cumulative weight lands in another slot than the
// reference's (about 10^4 of 2^24 copy_from entries per step with the
// reference's own weights and uniforms).  This file reproduces S_i bit for
// bit for non-negative weights:
//
// * While S_{i-1} and S_i lie in one binade [2^E, 2^(E+1)), both are
//   multiples of u = 2^(E-52), so S_i = S_{i-1} + k_i u with k_i = w_i / u
//   rounded to the nearest integer (a tie would depend on the last bit of
//   S_{i-1}).  Over a run of such "clean" elements the sum is an exact
//   integer sum.
// * An approximate prefix G_i with a proven error bound d_i decides which
//   elements are clean: the binade of G_{i-1} +- d and G_i +- d must be the
//   same.  |S_i - G_i| <= (i + 1) ulp(S_i) / 2 (each rounding of the
//   sequential sum) + the error of G (a relative margin of the weight
//   source); d_i = (8 i + 256) ulp(2 max(G, w)) + margin * max(G, w).
// * A zero weight while the prefix is still 0 leaves S at 0: clean, k = 0.
// * The other ("special") elements -- the first, binade crossings,
//   uncertain binades, ties -- are few (about 40 at N = 2^24): the spine
//   kernel visits them in order with one hardware addition each and jumps
//   over clean runs by their exact integer sums.
//
// Phase A (k_exact_tiles_body, per tile): classify, per-tile integer sums,
// the list of the tile's specials.  Phase B (k_exact_spine_body, one CTA):
// the exact S at every tile start and at every special.  Phase C (in
// k_invert_body): every element's S from its tile's start or its last
// special plus an integer prefix.  A tile with more than kExactCap specials
// (possible only for weights built to create ties) is summed element by
// element in phase B.
#pragma once

#include "smc_common.cuh"

namespace vsmc_b200 {

constexpr int kExactCap = 64;         // specials kept per tile
constexpr int kNoBinade = -100000;    // binade of a special element
constexpr int kExactStage = 1024;     // specials the spine stages

struct ExactTile {
    unsigned long long k_total; // sum of the clean elements' k
    int nspec;                  // specials of the tile
    int e_last;                 // binade of the last element (if clean)
};

struct ExactSpecial {
    double w;                     // the weight
    unsigned long long k_before;  // clean k of the tile before it
    int idx;                      // index in the tile
    int e_seg;                    // binade of the clean elements before it
};

// Device arrays of the exact scan (part of the resampling workspace).
struct ExactScan {
    ExactTile *tiles;       // ntiles
    ExactSpecial *spec;     // ntiles x kExactCap
    double *s_spec;         // ntiles x kExactCap: exact S at each special
    double *start;          // ntiles + 1: exact S before each tile (0 first)
    double *full;           // N: exact S of the elements of overflow tiles
    double *s_out;          // ntiles: exact S after each tile with specials
    unsigned long long *pk; // ntiles + 1: prefix of clean tiles' k_total
    int32_t *dirty;         // ntiles: the tiles with specials, in order
};

// Binade of a positive normal double: 2^E <= x < 2^(E+1).
__device__ __forceinline__ int exact_binade(double x)
{
    return (int)((__double_as_longlong(x) >> 52) & 0x7ff) - 1023;
}

// 2^e for -1022 <= e <= 1023.
__device__ __forceinline__ double exact_pow2(int e)
{
    return __longlong_as_double((long long)(e + 1023) << 52);
}

struct ExactElem {
    unsigned long long k;
    int e;
    bool special;
};

// Classification of element i with weight w, approximate prefixes gp
// (through i - 1) and g (through i), relative margin `rel` of the prefix.
__device__ __forceinline__ ExactElem exact_classify(long long i, double w,
                                                    double gp, double g,
                                                    double rel)
{
    ExactElem r;
    r.k = 0;
    r.e = kNoBinade;
    r.special = true;
    if (i == 0)
        return r; // S_{-1} = 0: the first addition is the hardware's
    if (gp == 0.0 && w == 0.0) {
        // a leading zero: every weight before it is 0 (sums of non-negative
        // weights vanish only so), S stays 0 and no k accumulates in its run
        r.special = false;
        return r;
    }
    const double m = fmax(fmax(g, gp), w);
    if (!(m > 0x1p-960 && m < 0x1p960) || !(w >= 0.0))
        return r;
    const double ulp2 = exact_pow2(exact_binade(m) + 1 - 52);
    const double d = __dadd_rn(__dmul_rn(__dadd_rn(8.0 * (double)i, 256.0),
                                         ulp2),
                               __dmul_rn(rel, m));
    const double plo = __dadd_rn(gp, -d);
    if (!(plo > 0x1p-960))
        return r;
    const double lo = __dadd_rn(g, -d), hi = __dadd_rn(g, d),
                 phi = __dadd_rn(gp, d);
    const int e = exact_binade(hi);
    if (exact_binade(lo) != e || exact_binade(plo) != e ||
        exact_binade(phi) != e)
        return r;
    // k = w / 2^(e-52), an exact scaling in two power-of-two steps
    const double kf = __dmul_rn(__dmul_rn(w, 0x1p52), exact_pow2(-e));
    if (!(kf < 0x1p52))
        return r;
    const double fl = floor(kf);
    if (__dadd_rn(kf, -fl) == 0.5)
        return r; // a tie: the rounding depends on the sum's last bit
    r.k = (unsigned long long)rint(kf);
    r.e = e;
    r.special = false;
    return r;
}

// The classification of a thread's kItems consecutive elements of a tile
// (global index i0 + j): approximate tile start `a`, the thread's exclusive
// prefix `pre` of the tile's weights, the weights `w`.  Elements at or past
// N count as clean with k = 0 and the previous element's binade.
struct ExactThread {
    unsigned long long kincl[kItems]; // clean k of the tile through j
    int e[kItems];
    unsigned special;                 // bit j
    int rank0;                        // specials of the tile before j = 0
    int nspec;                        // specials of the tile
    unsigned long long ktile;         // clean k of the tile
    int e_before;                     // binade of the element before j = 0
};

struct SmemExactThread {
    unsigned long long shk[kThreads / 32];
    int shi[kThreads / 32];
    int elast[kThreads];
};

__device__ __forceinline__ void
exact_thread(long long i0, long long N, const double (&w)[kItems], double a,
             double pre, double rel, ExactThread &x, SmemExactThread &sm)
{
    double gp = __dadd_rn(a, pre);
    double p = pre;
    unsigned long long kr = 0;
    int nsp = 0;
    int eprev = kNoBinade;
    unsigned long long kloc[kItems];
    x.special = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = i0 + j;
        p += w[j];
        const double g = __dadd_rn(a, p);
        if (i < N) {
            const ExactElem c = exact_classify(i, w[j], gp, g, rel);
            x.e[j] = c.e;
            if (c.special) {
                x.special |= 1u << j;
                ++nsp;
            }
            kr += c.k;
            eprev = c.e;
        } else {
            x.e[j] = eprev;
        }
        kloc[j] = kr;
        gp = g;
    }
    int nspec;
    x.rank0 = block_excl_scan(nsp, sm.shi, nspec);
    x.nspec = nspec;
    unsigned long long ktile;
    const unsigned long long kex = block_excl_scan(kr, sm.shk, ktile);
    x.ktile = ktile;
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        x.kincl[j] = kex + kloc[j];
    sm.elast[threadIdx.x] =
        (x.special >> (kItems - 1)) & 1u ? kNoBinade : x.e[kItems - 1];
    __syncthreads();
    x.e_before = threadIdx.x > 0 ? sm.elast[threadIdx.x - 1] : kNoBinade;
    __syncthreads();
}

// Phase A: one tile's classification, sums and specials.
__device__ __forceinline__ void
exact_tile_record(const ExactThread &x, const double (&w)[kItems],
                  long long base, long long i0, long long N, int tile,
                  const ExactScan &ex)
{
    int r = x.rank0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        if ((x.special >> j) & 1u) {
            if (r < kExactCap) {
                ExactSpecial s;
                s.w = w[j];
                s.k_before = x.kincl[j];
                s.idx = (int)(i0 + j - base);
                s.e_seg = j == 0 ? x.e_before
                                 : ((x.special >> (j - 1)) & 1u
                                        ? kNoBinade
                                        : x.e[j - 1]);
                ex.spec[(size_t)tile * kExactCap + r] = s;
            }
            ++r;
        }
    }
    const long long last = min(base + (long long)kTile, N) - 1;
    if (last >= i0 && last < i0 + kItems) {
        const int j = (int)(last - i0);
        ex.tiles[tile].e_last =
            (x.special >> j) & 1u ? kNoBinade : x.e[j];
    }
    if (threadIdx.x == 0) {
        ex.tiles[tile].k_total = x.ktile;
        ex.tiles[tile].nspec = x.nspec;
    }
}

// Phase C: the exact S of a thread's elements from the tile's exact start,
// its specials' exact values (staged: sv, kb for ranks < kExactCap) and,
// for an overflow tile, the element values phase B wrote.
__device__ __forceinline__ void
exact_values(const ExactThread &x, long long i0, double start,
             const double *sv, const unsigned long long *kb, bool overflow,
             const double *full, long long N, double (&S)[kItems])
{
    int r = x.rank0 - 1; // rank of the last special before element j
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = i0 + j;
        if (overflow) {
            S[j] = i < N ? full[i] : 0.0;
            continue;
        }
        // r < kExactCap holds when phases A and C classify alike (the same
        // arithmetic on the same inputs); the clamp keeps the read in bounds
        if ((x.special >> j) & 1u) {
            ++r;
            S[j] = sv[min(r, kExactCap - 1)];
        } else {
            const int rc = min(r, kExactCap - 1);
            const double b = r < 0 ? start : sv[rc];
            const unsigned long long k0 = r < 0 ? 0ull : kb[rc];
            const unsigned long long dk = x.kincl[j] - k0;
            S[j] = dk == 0 ? b
                           : __dadd_rn(b, __dmul_rn((double)dk,
                                                    exact_pow2(x.e[j] - 52)));
        }
    }
}

} // namespace vsmc_b200
