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
// * An approximate prefix G_i with a proven error bound d decides which
//   elements are clean: the windows G_{i-1} +- d and G_i +- d must lie in
//   one binade.  |S_i - G_i| <= (i + 1) ulp(S_i) / 2 (each rounding of the
//   sequential sum) + the error of G (a relative margin of the weight
//   source); each thread uses one bound for its kItems elements,
//   d = (8 i_last + 256) ulp(2 m) + margin * m, m >= every G and w there.
// * A zero weight while the prefix is still 0 leaves S at 0: clean, k = 0.
// * The other ("special") elements -- the first, binade crossings,
//   uncertain binades, ties -- are few (about 40 at N = 2^24): the spine
//   kernel visits them in order with one hardware addition each and jumps
//   over clean runs by their exact integer sums.
//
// Phase A (k_exact_tiles_body, per tile): classify, per-tile integer sums,
// the list of the tile's specials and, per element, a record: the exact
// offset of S_i from the S of the tile's last special before it (or of the
// tile's start), or -1 at a special.  Phase B (k_exact_spine_body, one CTA):
// the exact S at every tile start and at every special.  Phase C (in
// k_invert_body): S_i = base + record, one exact addition, with no weight,
// exp or classification.  A tile with more than kExactCap specials
// (possible only for weights built to create ties) is summed element by
// element in phase B, which writes S_i itself into its records.
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
    double *rec;            // N: per-element record (see above)
    int32_t *kint;          // N: floor(N w) (residual schemes)
    // per tile with specials, by rank (those past the spine's shared stage)
    double *s_out;          // exact S after the tile
    unsigned long long *pk; // clean k before the tile
    int32_t *dirty;         // the tile
    int32_t *eaft;          // binade of the clean tiles after it
};

// Binade of a positive normal double: 2^E <= x < 2^(E+1).
__device__ __forceinline__ int exact_binade(double x)
{
    return ((__double2hiint(x) >> 20) & 0x7ff) - 1023;
}

// 2^e for -1022 <= e <= 1023.
__device__ __forceinline__ double exact_pow2(int e)
{
    return __hiloint2double((e + 1023) << 20, 0);
}

// Binade shared by every value of [g - d, g + d], or kNoBinade.
__device__ __forceinline__ int exact_window(double g, double d)
{
    const double lo = __dadd_rn(g, -d), hi = __dadd_rn(g, d);
    if (!(lo > 0x1p-960))
        return kNoBinade;
    const int e = exact_binade(hi);
    return exact_binade(lo) == e ? e : kNoBinade;
}

// Block-wide exclusive max-scan of one value per thread (0 before the
// first); `sh` needs blockDim.x/32 entries.
__device__ __forceinline__ unsigned long long
block_excl_max(unsigned long long v, unsigned long long *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    unsigned long long inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long n = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
            inc = max(inc, n);
    }
    if (lane == 31)
        sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        unsigned long long s = lane < nw ? sh[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long n = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o)
                s = max(s, n);
        }
        if (lane < nw)
            sh[lane] = s;
    }
    __syncthreads();
    unsigned long long ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0)
        ex = 0;
    if (wid > 0)
        ex = max(ex, sh[wid - 1]);
    __syncthreads();
    return ex;
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
    unsigned long long kb_in;         // kincl at the tile's last special
                                      // before j = 0 (0: none)
    int e_before;                     // binade of the element before j = 0
};

struct SmemExactThread {
    unsigned long long shk[kThreads / 32];
    unsigned long long shm[kThreads / 32];
    int shi[kThreads / 32];
    int elast[kThreads];
};

__device__ __forceinline__ void
exact_thread(long long i0, long long N, const double (&w)[kItems], double a,
             double pre, double rel, ExactThread &x, SmemExactThread &sm)
{
    // one error bound for the thread's elements
    double p = pre, wmax = 0.0;
    bool bad = false;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        p += w[j];
        wmax = fmax(wmax, w[j]);
        bad |= !(w[j] >= 0.0);
    }
    const double m = fmax(__dadd_rn(a, p), wmax);
    const bool ok = !bad && m > 0x1p-960 && m < 0x1p960;
    double d = 0.0;
    if (ok) {
        const double ulp2 = exact_pow2(exact_binade(m) + 1 - 52);
        const double il = (double)(i0 + kItems - 1);
        d = __dadd_rn(__dmul_rn(__dadd_rn(8.0 * il, 256.0), ulp2),
                      __dmul_rn(rel, m));
    }
    double gp = __dadd_rn(a, pre);
    unsigned long long kr = 0;
    int nsp = 0;
    unsigned long long kloc[kItems];
    x.special = 0;
    // the common case: the windows of the thread's first and last prefix
    // lie in one binade, so every window between them does and each of
    // the thread's elements is clean (unless a tie)
    bool fast = false;
    if (ok && i0 > 0 && i0 + kItems <= N) {
        const int e0 = exact_window(gp, d);
        if (e0 != kNoBinade && e0 == exact_window(__dadd_rn(a, p), d)) {
            const double sc = exact_pow2(52 - e0);
            bool slow = false;
#pragma unroll
            for (int j = 0; j < kItems; ++j) {
                const double kf = __dmul_rn(w[j], sc);
                const double t = __dadd_rn(kf, 0x1p52);
                slow |= !(kf < 0x1p52) ||
                        fabs(__dadd_rn(__dadd_rn(t, -0x1p52), -kf)) == 0.5;
                kr += (unsigned long long)(__double_as_longlong(t) -
                                           __double_as_longlong(0x1p52));
                kloc[j] = kr;
                x.e[j] = e0;
            }
            fast = !slow;
        }
    }
    int ep = ok && !fast ? exact_window(gp, d) : kNoBinade;
    p = pre;
    int eprev = kNoBinade;
    if (!fast) {
        kr = 0;
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const long long i = i0 + j;
            p += w[j];
            const double g = __dadd_rn(a, p);
            const int ec = ok ? exact_window(g, d) : kNoBinade;
            if (i < N) {
                bool sp = true;
                unsigned long long k = 0;
                int e = kNoBinade;
                if (i == 0) {
                    // S_{-1} = 0: the first addition is the hardware's
                } else if (gp == 0.0 && w[j] == 0.0) {
                    // a leading zero: every weight before it is 0 (sums of
                    // non-negative weights vanish only so)
                    sp = false;
                } else if (ec != kNoBinade && ec == ep) {
                    // k = w / 2^(e-52) rounded to nearest: adding 2^52 rounds
                    // it to an integer; a tie depends on the sum's last bit
                    const double kf = __dmul_rn(w[j], exact_pow2(52 - ec));
                    if (kf < 0x1p52) {
                        const double t = __dadd_rn(kf, 0x1p52);
                        const double kd = __dadd_rn(t, -0x1p52);
                        if (fabs(__dadd_rn(kd, -kf)) != 0.5) {
                            k = (unsigned long long)(__double_as_longlong(t) -
                                                     __double_as_longlong(0x1p52));
                            e = ec;
                            sp = false;
                        }
                    }
                }
                x.e[j] = e;
                if (sp) {
                    x.special |= 1u << j;
                    ++nsp;
                }
                kr += k;
                eprev = e;
            } else {
                x.e[j] = eprev;
            }
            kloc[j] = kr;
            gp = g;
            ep = ec;
        }
    }
    int nspec;
    x.rank0 = block_excl_scan(nsp, sm.shi, nspec);
    x.nspec = nspec;
    unsigned long long ktile;
    const unsigned long long kex = block_excl_scan(kr, sm.shk, ktile);
    x.ktile = ktile;
    unsigned long long vlast = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        x.kincl[j] = kex + kloc[j];
        if ((x.special >> j) & 1u)
            vlast = x.kincl[j];
    }
    // kincl is non-decreasing, so the last special before the chunk holds
    // the largest kincl of the earlier threads' last specials
    x.kb_in = block_excl_max(vlast, sm.shm);
    sm.elast[threadIdx.x] =
        (x.special >> (kItems - 1)) & 1u ? kNoBinade : x.e[kItems - 1];
    __syncthreads();
    x.e_before = threadIdx.x > 0 ? sm.elast[threadIdx.x - 1] : kNoBinade;
    __syncthreads();
}

// Phase A: one tile's specials and sums, and the thread's element records
// (the exact offset from the base, -1 at a special) into `rec`.
__device__ __forceinline__ void
exact_tile_record(const ExactThread &x, const double (&w)[kItems],
                  long long base, long long i0, long long N, int tile,
                  const ExactScan &ex, double (&rec)[kItems])
{
    int r = x.rank0;
    unsigned long long kb = x.kb_in;
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
            kb = x.kincl[j];
            rec[j] = -1.0;
        } else {
            const unsigned long long K = x.kincl[j] - kb;
            rec[j] = K == 0 ? 0.0
                            : __dmul_rn((double)K, exact_pow2(x.e[j] - 52));
        }
    }
    const long long last = min(base + (long long)kTile, N) - 1;
#pragma unroll
    for (int j = 0; j < kItems; ++j) // (constant indices keep x in registers)
        if (i0 + j == last)
            ex.tiles[tile].e_last =
                (x.special >> j) & 1u ? kNoBinade : x.e[j];
    if (threadIdx.x == 0) {
        ex.tiles[tile].k_total = x.ktile;
        ex.tiles[tile].nspec = x.nspec;
    }
}

// Phase C: the exact S of a thread's elements from their records, the
// tile's exact start and its specials' exact values sv (ranks below
// kExactCap); an overflow tile's records hold S itself.
__device__ __forceinline__ void
exact_values(const double (&rec)[kItems], int rank0, double start,
             const double *sv, bool overflow, double (&S)[kItems])
{
    int r = rank0 - 1; // rank of the last special before element j
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        if (overflow) {
            S[j] = rec[j];
            continue;
        }
        // r < kExactCap holds when the records and the specials come from
        // one classification; the clamp keeps the read in bounds
        if (rec[j] < 0.0) {
            ++r;
            S[j] = sv[min(r, kExactCap - 1)];
        } else {
            const double b = r < 0 ? start : sv[min(r, kExactCap - 1)];
            S[j] = __dadd_rn(b, rec[j]);
        }
    }
}

} // namespace vsmc_b200
