/*
 * smc_oracle.c -- CPU restatement of vSMC's SMC step (TEST INFRASTRUCTURE).
 *
 * Checker only: loaded by tests/, __graft_entry__.smoke() and bench.py's CPU
 * legs; never linked into the product.  Build flags (oracle/Makefile):
 * -O2 -ffp-contract=off, no -march, so every double operation below is the
 * single IEEE operation the reference's C++ performs, in the same order.
 * Citations are relative to the vSMC project root.
 */
#include "smc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------ Philox -- */

/* Weyl key bumps and round multipliers: include/vsmc/rng/philox.hpp:77-103
 * (PHILOX_W32_0/1 and PHILOX_M4x32_0/1 of the Random123 paper). */
#define ORC_PHILOX_W0 0x9E3779B9u
#define ORC_PHILOX_W1 0xBB67AE85u
#define ORC_PHILOX_M0 0xD2511F53u
#define ORC_PHILOX_M1 0xCD9E8D57u

void orc_philox4x32_block(const uint32_t ctr[4], const uint32_t key[2],
                          uint32_t out[4])
{
    /* generate_buffer (philox.hpp:504-523): rounds N = 1..10; the key is
     * bumped before every round but the first (PhiloxBumpKey, :137-160);
     * each round is PhiloxRound<uint32_t,4> (:231-265). */
    uint32_t s0 = ctr[0], s1 = ctr[1], s2 = ctr[2], s3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 1; r <= 10; ++r) {
        if (r > 1) {
            k0 += ORC_PHILOX_W0;
            k1 += ORC_PHILOX_W1;
        }
        uint64_t pa = (uint64_t)ORC_PHILOX_M1 * (uint64_t)s2; /* hi0, lo1 */
        uint64_t pb = (uint64_t)ORC_PHILOX_M0 * (uint64_t)s0; /* hi2, lo3 */
        uint32_t hi0 = (uint32_t)(pa >> 32) ^ k0;
        uint32_t lo1 = (uint32_t)pa;
        uint32_t hi2 = (uint32_t)(pb >> 32) ^ k1;
        uint32_t lo3 = (uint32_t)pb;
        s0 = hi0 ^ s1;
        s1 = lo1;
        s2 = hi2 ^ s3;
        s3 = lo3;
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
    out[3] = s3;
}

/* ---------------------------------------------------------- Threefry -- */

/* Key-schedule parity constant: threefry.hpp:65-73 (SKEIN_KS_PARITY). */
#define ORC_THREEFRY_KS 0x1BD11BDAA9FC1A22ull

/* Rotation constants for 4x64, by (round-1)%8 and pair: threefry.hpp:105-130
 * (the Threefish-256 rotation table). */
static const unsigned orc_tf_rot[8][2] = {
    {14, 16}, {52, 57}, {23, 40}, {5, 37},
    {25, 33}, {46, 12}, {58, 22}, {32, 32}};

static uint64_t orc_rotl64(uint64_t x, unsigned r)
{
    return (x << r) | (x >> (64 - r));
}

void orc_threefry4x64_block(const uint64_t ctr[4], const uint64_t key[4],
                            uint64_t out[4])
{
    /* init_par (threefry.hpp:491-506): par[0..3] = key, par[4] = KS ^ k0 ^
     * k1 ^ k2 ^ k3. */
    uint64_t par[5];
    par[4] = ORC_THREEFRY_KS;
    for (int i = 0; i != 4; ++i) {
        par[i] = key[i];
        par[4] ^= key[i];
    }
    uint64_t b[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    /* generate_buffer (:473-489): for N = 0..20, ThreefryRotate (no-op at
     * N = 0; pairs (0,i0),(2,i2) with i0 = N odd ? 1 : 3, :142-185) then
     * ThreefryInsertKey when N % 4 == 0 (inc = N/4 added to word 3 after the
     * key words par[(inc+j)%5], :187-233). */
    for (unsigned n = 0; n <= 20; ++n) {
        if (n > 0) {
            const unsigned r = (n - 1) % 8;
            const int i0 = (n % 2) ? 1 : 3;
            const int i2 = (n % 2) ? 3 : 1;
            b[0] += b[i0];
            b[i0] = orc_rotl64(b[i0], orc_tf_rot[r][0]);
            b[i0] ^= b[0];
            b[2] += b[i2];
            b[i2] = orc_rotl64(b[i2], orc_tf_rot[r][1]);
            b[i2] ^= b[2];
        }
        if (n % 4 == 0) {
            const unsigned inc = n / 4;
            for (unsigned j = 0; j != 4; ++j)
                b[j] += par[(inc + j) % 5];
            b[3] += inc;
        }
    }
    for (int i = 0; i != 4; ++i)
        out[i] = b[i];
}

/* ------------------------------------------------------------ engines -- */

/* Counter<Array<T,K>>::increment (utility/counter.hpp:119-120, 180-192):
 * little-endian add with carry starting at word 0. */
static void orc_ctr_inc32(uint32_t c[4])
{
    for (int i = 0; i != 4; ++i)
        if (++c[i] != 0)
            return;
}

static void orc_ctr_inc64(uint64_t c[4])
{
    for (int i = 0; i != 4; ++i)
        if (++c[i] != 0)
            return;
}

void orc_philox_seed(orc_philox *e, uint32_t s)
{
    memset(e->ctr, 0, sizeof(e->ctr));
    e->key[0] = s;
    e->key[1] = 0;
    e->index = 4;
}

void orc_threefry_seed(orc_threefry *e, uint64_t s)
{
    memset(e->ctr, 0, sizeof(e->ctr));
    e->key[0] = s;
    e->key[1] = e->key[2] = e->key[3] = 0;
    e->index = 4;
}

void orc_philox_set_key(orc_philox *e, const uint32_t key[2])
{
    e->key[0] = key[0];
    e->key[1] = key[1];
    e->index = 4;
}

void orc_philox_set_ctr(orc_philox *e, const uint32_t ctr[4])
{
    memcpy(e->ctr, ctr, sizeof(e->ctr));
    e->index = 4;
}

void orc_threefry_set_key(orc_threefry *e, const uint64_t key[4])
{
    memcpy(e->key, key, sizeof(e->key));
    e->index = 4;
}

void orc_threefry_set_ctr(orc_threefry *e, const uint64_t ctr[4])
{
    memcpy(e->ctr, ctr, sizeof(e->ctr));
    e->index = 4;
}

uint32_t orc_philox_next(orc_philox *e)
{
    if (e->index == 4) {
        orc_ctr_inc32(e->ctr);
        orc_philox4x32_block(e->ctr, e->key, e->buf);
        e->index = 0;
    }
    return e->buf[e->index++];
}

uint64_t orc_threefry_next(orc_threefry *e)
{
    if (e->index == 4) {
        orc_ctr_inc64(e->ctr);
        orc_threefry4x64_block(e->ctr, e->key, e->buf);
        e->index = 0;
    }
    return e->buf[e->index++];
}

uint64_t orc_threefry_words_used(const orc_threefry *e)
{
    if (e->ctr[0] == 0)
        return 0;
    return (e->ctr[0] - 1) * 4 + e->index;
}

/* Word w (0-based) after ctr0 with an empty buffer is lane w % 4 of block
 * ctr0 + w/4 + 1 (increment-before-generate). */
static void orc_ctr_add32(uint32_t c[4], uint64_t v)
{
    uint64_t carry = v;
    for (int i = 0; i != 4 && carry; ++i) {
        uint64_t s = (uint64_t)c[i] + (carry & 0xFFFFFFFFull);
        c[i] = (uint32_t)s;
        carry = (carry >> 32) + (s >> 32);
    }
}

static void orc_ctr_add64(uint64_t c[4], uint64_t v)
{
    uint64_t carry = v;
    for (int i = 0; i != 4 && carry; ++i) {
        uint64_t s = c[i] + carry;
        carry = (s < c[i]) ? 1 : 0;
        c[i] = s;
    }
}

void orc_philox_stream(const uint32_t key[2], const uint32_t ctr0[4],
                       uint64_t skip, uint64_t n, uint32_t *out)
{
    uint32_t blk[4] = {0, 0, 0, 0};
    uint64_t cur = UINT64_MAX;
    for (uint64_t k = 0; k != n; ++k) {
        const uint64_t w = skip + k;
        if (w / 4 != cur) {
            uint32_t c[4] = {ctr0[0], ctr0[1], ctr0[2], ctr0[3]};
            orc_ctr_add32(c, w / 4 + 1);
            orc_philox4x32_block(c, key, blk);
            cur = w / 4;
        }
        out[k] = blk[w % 4];
    }
}

void orc_threefry_stream(const uint64_t key[4], const uint64_t ctr0[4],
                         uint64_t skip, uint64_t n, uint64_t *out)
{
    uint64_t blk[4] = {0, 0, 0, 0};
    uint64_t cur = UINT64_MAX;
    for (uint64_t k = 0; k != n; ++k) {
        const uint64_t w = skip + k;
        if (w / 4 != cur) {
            uint64_t c[4] = {ctr0[0], ctr0[1], ctr0[2], ctr0[3]};
            orc_ctr_add64(c, w / 4 + 1);
            orc_threefry4x64_block(c, key, blk);
            cur = w / 4;
        }
        out[k] = blk[w % 4];
    }
}

/* --------------------------------------------------------------- U01 -- */

double orc_u01_closed_open_64_53(uint64_t u)
{
    return (double)(u >> 11) * 0x1p-53; /* u01.h:151-153 */
}

double orc_u01_open_closed_32_53(uint32_t u)
{
    return (1.0 + (double)u) * 0x1p-32; /* u01.h:124-126 */
}

/* libstdc++ generate_canonical<double, 53> (bits/random.tcc): k words,
 * sum += double(word) * 2^(32*j), result sum / 2^(wordbits*k), and a result
 * of 1 is replaced by nextafter(1, 0). */
double orc_canonical_u64(uint64_t x)
{
    double sum = (double)x;
    double r = sum / 18446744073709551616.0;
    if (r >= 1.0)
        r = nextafter(1.0, 0.0);
    return r;
}

double orc_canonical_u32x2(uint32_t a, uint32_t b)
{
    double sum = (double)a;
    sum = sum + (double)b * 4294967296.0;
    double r = sum / 18446744073709551616.0;
    if (r >= 1.0)
        r = nextafter(1.0, 0.0);
    return r;
}

void orc_normal_reset(orc_normal *nd)
{
    nd->saved_available = 0;
    nd->saved = 0;
}

/* Marsaglia polar method as libstdc++'s normal_distribution::operator()
 * applies it: x, y = 2U - 1 from two canonical draws; reject r2 > 1 or
 * r2 == 0; mult = sqrt(-2 log(r2) / r2); cache x*mult, return y*mult;
 * then ret * sd + mean. */
double orc_normal_philox(orc_normal *nd, orc_philox *e, double mean, double sd)
{
    double ret;
    if (nd->saved_available) {
        nd->saved_available = 0;
        ret = nd->saved;
    } else {
        double x, y, r2;
        do {
            uint32_t a = orc_philox_next(e);
            uint32_t b = orc_philox_next(e);
            x = 2.0 * orc_canonical_u32x2(a, b) - 1.0;
            a = orc_philox_next(e);
            b = orc_philox_next(e);
            y = 2.0 * orc_canonical_u32x2(a, b) - 1.0;
            r2 = x * x + y * y;
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = sqrt(-2.0 * log(r2) / r2);
        nd->saved = x * mult;
        nd->saved_available = 1;
        ret = y * mult;
    }
    return ret * sd + mean;
}

/* ----------------------------------------------------------- weights -- */

static double orc_post_set_log_weight(size_t N, double *lw, double *w)
{
    /* normalize_log_weight (weight_set.hpp:108-117) */
    double dmax = lw[0];
    for (size_t i = 0; i != N; ++i)
        if (dmax < lw[i])
            dmax = lw[i];
    dmax = -dmax;
    for (size_t i = 0; i != N; ++i)
        lw[i] += dmax;
    /* log_weight2weight = vExp (:369-370, math/vmath.hpp:45-52) */
    for (size_t i = 0; i != N; ++i)
        w[i] = exp(lw[i]);
    /* normalize_weight (:119-125): coeff = 1/asum, scal, ess = 1/dot */
    double sum = 0;
    for (size_t i = 0; i != N; ++i)
        sum += fabs(w[i]);
    const double coeff = 1 / sum;
    for (size_t i = 0; i != N; ++i)
        w[i] *= coeff;
    double dot = 0;
    for (size_t i = 0; i != N; ++i)
        dot = dot + w[i] * w[i];
    return 1 / dot;
}

double orc_add_log_weight(size_t N, double *lw, double *w, const double *inc)
{
    if (inc != NULL)
        for (size_t i = 0; i != N; ++i)
            lw[i] += inc[i];
    return orc_post_set_log_weight(N, lw, w);
}

double orc_set_equal_weight(size_t N, double *lw, double *w)
{
    const double ess = (double)N;
    for (size_t i = 0; i != N; ++i) {
        w[i] = 1 / ess;
        lw[i] = 0;
    }
    return ess;
}

/* ---------------------------------------------------------- resample -- */

/* The three lazily evaluated U01 sequences of rng/u01.hpp:165-287. */
typedef struct {
    int kind; /* 0 sorted, 1 stratified, 2 systematic, 3 given */
    size_t N, n;
    double u, lmax, u0, delta;
    orc_threefry *rng;
    const double *given;
    double *log;
    size_t nlog;
} orc_u01seq;

static void orc_u01seq_init(orc_u01seq *s, int kind, size_t N,
                            orc_threefry *rng, double *log)
{
    memset(s, 0, sizeof(*s));
    s->kind = kind;
    s->N = N;
    s->n = N;
    s->u = 0;
    s->lmax = 0;
    s->rng = rng;
    s->log = log;
    s->delta = 1.0 / (double)N;
    if (kind == 2) /* U01SequenceSystematic ctor draws u0 at once (:258-263) */
        s->u0 = orc_canonical_u64(orc_threefry_next(rng)) * s->delta;
}

static double orc_u01seq_at(orc_u01seq *s, size_t n)
{
    if (n == s->n)
        return s->u;
    switch (s->kind) {
    case 0: /* sorted (:182-189) */
        s->lmax += log(1 - orc_canonical_u64(orc_threefry_next(s->rng))) /
                   (double)(s->N - n);
        s->n = n;
        s->u = 1 - exp(s->lmax);
        break;
    case 1: /* stratified (:224-230) */
        s->n = n;
        s->u = orc_canonical_u64(orc_threefry_next(s->rng)) * s->delta +
               (double)n * s->delta;
        break;
    case 2: /* systematic (:271-276) */
        s->n = n;
        s->u = s->u0 + (double)n * s->delta;
        break;
    default:
        s->n = n;
        s->u = s->given[n];
        break;
    }
    if (s->log != NULL)
        s->log[s->nlog] = s->u;
    s->nlog++;
    return s->u;
}

/* internal::inversion (resample/common.hpp:57-84) */
static void orc_inversion_seq(size_t M, size_t N, const double *weight,
                              orc_u01seq *seq, int64_t *rep)
{
    if (M == 0)
        return;
    if (M == 1) {
        rep[0] = (int64_t)N;
        return;
    }
    memset(rep, 0, sizeof(int64_t) * M);
    if (N == 0)
        return;
    size_t n = 0;
    double accw = 0;
    for (size_t i = 0; i != M - 1; ++i) {
        accw += weight[i];
        while (n != N && orc_u01seq_at(seq, n) <= accw) {
            ++rep[i];
            ++n;
        }
    }
    rep[M - 1] = (int64_t)(N - n);
}

void orc_inversion(size_t M, size_t N, const double *weight, const double *u,
                   int64_t *replication)
{
    orc_u01seq s;
    memset(&s, 0, sizeof(s));
    s.kind = 3;
    s.N = N;
    s.n = N;
    s.given = u;
    orc_inversion_seq(M, N, weight, &s, replication);
}

void orc_resample(int scheme, size_t M, size_t N, orc_threefry *rng,
                  const double *weight, int64_t *rep, double *uniforms,
                  size_t *n_uniforms)
{
    orc_u01seq s;
    int kind = 0;
    switch (scheme) {
    case ORC_MULTINOMIAL:
    case ORC_RESIDUAL:
        kind = 0;
        break;
    case ORC_STRATIFIED:
    case ORC_RESIDUAL_STRATIFIED:
        kind = 1;
        break;
    default:
        kind = 2;
        break;
    }
    if (scheme == ORC_MULTINOMIAL || scheme == ORC_STRATIFIED ||
        scheme == ORC_SYSTEMATIC) {
        orc_u01seq_init(&s, kind, N, rng, uniforms);
        orc_inversion_seq(M, N, weight, &s, rep);
    } else {
        /* residual.hpp:59-76: r = modf(N w, &k); r *= 1/asum(r);
         * NN = N - sum k; inversion of NN on r; rep += k. */
        double *r = (double *)malloc(sizeof(double) * (M ? M : 1));
        double *k = (double *)malloc(sizeof(double) * (M ? M : 1));
        for (size_t i = 0; i != M; ++i)
            r[i] = modf((double)N * weight[i], k + i);
        double sum = 0;
        for (size_t i = 0; i != M; ++i)
            sum += fabs(r[i]);
        const double coeff = 1 / sum;
        for (size_t i = 0; i != M; ++i)
            r[i] *= coeff;
        int64_t R = 0;
        for (size_t i = 0; i != M; ++i)
            R += (int64_t)k[i];
        const size_t NN = N - (size_t)R;
        orc_u01seq_init(&s, kind, NN, rng, uniforms);
        orc_inversion_seq(M, NN, r, &s, rep);
        for (size_t i = 0; i != M; ++i)
            rep[i] += (int64_t)k[i];
        free(r);
        free(k);
    }
    if (n_uniforms != NULL)
        *n_uniforms = s.nlog;
}

/* internal::cfrp_trans (resample/common.hpp:87-118) */
void orc_cfrp_trans(size_t M, size_t N, const int64_t *rep,
                    int64_t *copy_from)
{
    if (M == N) {
        int64_t time = 0;
        int64_t from = 0;
        for (size_t to = 0; to != N; ++to) {
            if (rep[to] != 0) {
                copy_from[to] = (int64_t)to;
            } else {
                if (rep[from] < time + 2) {
                    time = 0;
                    do
                        ++from;
                    while (rep[from] < 2);
                }
                copy_from[to] = from;
                ++time;
            }
        }
    } else {
        size_t to = 0;
        for (size_t from = 0; from != M; ++from)
            for (int64_t r = 0; r != rep[from]; ++r)
                copy_from[to++] = (int64_t)from;
    }
}

/* ---------------------------------------------------------- CV model -- */

void orc_cv_default(orc_cv_param *p)
{
    p->dt = 0.1;
    p->sd_pos = 0.02;
    p->sd_vel = 0.5;
    p->sd_pos0 = 2;
    p->sd_vel0 = 1;
    p->scale = 10;
    p->nu = 10;
}

/* cv_state::log_likelihood (example/pf/include/pf_smp.hpp:96-112) */
double orc_cv_loglik(const orc_cv_param *p, double x, double y, double ox,
                     double oy)
{
    double llh_x = p->scale * (x - ox);
    double llh_y = p->scale * (y - oy);
    llh_x = log(1 + llh_x * llh_x / p->nu);
    llh_y = log(1 + llh_y * llh_y / p->nu);
    return -0.5 * (p->nu + 1) * (llh_x + llh_y);
}

/* cv_init::initialize_state (pf_smp.hpp:150-173) */
void orc_cv_init_particle(const orc_cv_param *p, const uint32_t key[2],
                          uint32_t id, uint32_t stream, double s[4])
{
    orc_philox e;
    const uint32_t ctr[4] = {0, 0, id, stream};
    orc_philox_set_key(&e, key);
    orc_philox_set_ctr(&e, ctr);
    orc_normal np, nv;
    orc_normal_reset(&np);
    orc_normal_reset(&nv);
    s[0] = orc_normal_philox(&np, &e, 0, p->sd_pos0);
    s[1] = orc_normal_philox(&np, &e, 0, p->sd_pos0);
    s[2] = orc_normal_philox(&nv, &e, 0, p->sd_vel0);
    s[3] = orc_normal_philox(&nv, &e, 0, p->sd_vel0);
}

/* cv_move::move_state (pf_smp.hpp:207-238) */
void orc_cv_move_particle(const orc_cv_param *p, const uint32_t key[2],
                          uint32_t iter, uint32_t id, uint32_t stream,
                          double s[4])
{
    orc_philox e;
    const uint32_t ctr[4] = {0, iter, id, stream};
    orc_philox_set_key(&e, key);
    orc_philox_set_ctr(&e, ctr);
    orc_normal np, nv;
    orc_normal_reset(&np);
    orc_normal_reset(&nv);
    double n;
    n = orc_normal_philox(&np, &e, 0, p->sd_pos);
    s[0] += n + p->dt * s[2];
    n = orc_normal_philox(&np, &e, 0, p->sd_pos);
    s[1] += n + p->dt * s[3];
    n = orc_normal_philox(&nv, &e, 0, p->sd_vel);
    s[2] += n;
    n = orc_normal_philox(&nv, &e, 0, p->sd_vel);
    s[3] += n;
}

static double orc_student_t(orc_normal *nd, orc_philox *e, double nu)
{
    const double z0 = orc_normal_philox(nd, e, 0, 1);
    const int k = (int)nu;
    double chi = 0;
    for (int i = 0; i != k; ++i) {
        const double z = orc_normal_philox(nd, e, 0, 1);
        chi += z * z;
    }
    return z0 / sqrt(chi / nu);
}

void orc_cv_simulate(const orc_cv_param *p, uint32_t obs_seed,
                     uint32_t stream, size_t T, double *obs_x, double *obs_y,
                     double *truth)
{
    double s[4] = {0, 0, 1, 1};
    const uint32_t key[2] = {obs_seed, 1};
    for (size_t t = 0; t != T; ++t) {
        orc_philox e;
        const uint32_t ctr[4] = {0, (uint32_t)t, 0, stream};
        orc_philox_set_key(&e, key);
        orc_philox_set_ctr(&e, ctr);
        orc_normal nd;
        orc_normal_reset(&nd);
        if (t > 0) {
            double n;
            n = orc_normal_philox(&nd, &e, 0, p->sd_pos);
            s[0] += n + p->dt * s[2];
            n = orc_normal_philox(&nd, &e, 0, p->sd_pos);
            s[1] += n + p->dt * s[3];
            n = orc_normal_philox(&nd, &e, 0, p->sd_vel);
            s[2] += n;
            n = orc_normal_philox(&nd, &e, 0, p->sd_vel);
            s[3] += n;
        }
        const double tx = orc_student_t(&nd, &e, p->nu);
        const double ty = orc_student_t(&nd, &e, p->nu);
        obs_x[t] = s[0] + tx / p->scale;
        obs_y[t] = s[1] + ty / p->scale;
        if (truth != NULL)
            for (int d = 0; d != 4; ++d)
                truth[t * 4 + d] = s[d];
    }
}

/* Seed::get(): skip() then return the internal seed (rng/seed.hpp:102,149,
 * with seed_max = 2^32-1 for the default unsigned result type). */
static uint32_t orc_seed_next(uint32_t *seed)
{
    *seed = (*seed == 0xFFFFFFFFu) ? 1u : (*seed + 1u);
    return *seed;
}

double orc_cv_filter(const orc_cv_param *p, size_t N, size_t T, int scheme,
                     double threshold, uint32_t seed, uint32_t stream,
                     const double *obs_x, const double *obs_y,
                     orc_cv_out *out)
{
    uint32_t sg = seed % 0xFFFFFFFFu; /* SeedGenerator::set */
    const uint32_t model_seed = orc_seed_next(&sg);
    const uint32_t resample_seed = orc_seed_next(&sg);
    const uint32_t key[2] = {model_seed, 0};
    orc_threefry rrng;
    orc_threefry_seed(&rrng, resample_seed);

    double *st = (double *)malloc(sizeof(double) * 4 * N);
    double *tmp = (double *)malloc(sizeof(double) * 4 * N);
    double *lw = (double *)malloc(sizeof(double) * N);
    double *w = (double *)malloc(sizeof(double) * N);
    double *inc = (double *)malloc(sizeof(double) * N);
    int64_t *rep = (int64_t *)malloc(sizeof(int64_t) * N);
    int64_t *cf = (int64_t *)malloc(sizeof(int64_t) * N);

    double logz = 0;
    double ess = orc_set_equal_weight(N, lw, w); /* do_reset */
    for (size_t t = 0; t != T; ++t) {
        /* move (or init at t = 0); the estimator reads W before the add */
        for (size_t i = 0; i != N; ++i) {
            double s[4];
            if (t == 0) {
                orc_cv_init_particle(p, key, (uint32_t)i, stream, s);
            } else {
                for (int d = 0; d != 4; ++d)
                    s[d] = st[d * N + i];
                orc_cv_move_particle(p, key, (uint32_t)t, (uint32_t)i,
                                     stream, s);
            }
            for (int d = 0; d != 4; ++d)
                st[d * N + i] = s[d];
            inc[i] = orc_cv_loglik(p, s[0], s[1], obs_x[t], obs_y[t]);
        }
        double sum = 0;
        for (size_t i = 0; i != N; ++i)
            sum += w[i] * exp(inc[i]);
        const double dz = log(sum);
        logz += dz;
        if (t == 0) {
            for (size_t i = 0; i != N; ++i)
                lw[i] = inc[i];
            ess = orc_add_log_weight(N, lw, w, NULL);
        } else {
            ess = orc_add_log_weight(N, lw, w, inc);
        }
        /* do_resample (sampler.hpp:816-822) -> Particle::resample
         * (particle.hpp:230-250) */
        int resampled = ess < threshold * (double)N;
        if (out && out->ess)
            out->ess[t] = ess;
        if (out && out->logz_inc)
            out->logz_inc[t] = dz;
        if (resampled) {
            orc_resample(scheme, N, N, &rrng, w, rep, NULL, NULL);
            orc_cfrp_trans(N, N, rep, cf);
            for (size_t to = 0; to != N; ++to)
                for (int d = 0; d != 4; ++d)
                    tmp[d * N + to] = st[d * N + (size_t)cf[to]];
            memcpy(st, tmp, sizeof(double) * 4 * N);
            ess = orc_set_equal_weight(N, lw, w);
            if (out && out->last_copy_from)
                memcpy(out->last_copy_from, cf, sizeof(int64_t) * N);
        }
        if (out && out->resampled)
            out->resampled[t] = resampled;
        /* Monitor at MonitorMCMC: ISIntegrate (integrate/is_integrate.hpp:
         * 56-80, non-CBLAS loop) of (x, y) against the normalised weights */
        double ex = 0, ey = 0;
        for (size_t i = 0; i != N; ++i) {
            ex += w[i] * st[i];
            ey += w[i] * st[N + i];
        }
        if (out && out->mean_x)
            out->mean_x[t] = ex;
        if (out && out->mean_y)
            out->mean_y[t] = ey;
    }
    if (out && out->final_state)
        memcpy(out->final_state, st, sizeof(double) * 4 * N);
    if (out && out->final_lw)
        memcpy(out->final_lw, lw, sizeof(double) * N);
    if (out && out->words_used)
        *out->words_used = orc_threefry_words_used(&rrng);
    free(st);
    free(tmp);
    free(lw);
    free(w);
    free(inc);
    free(rep);
    free(cf);
    return logz;
}
