/*
 * ORACLE -- test infrastructure only.
 * Philox4x64-10 streams (Salmon et al., SC 2011) with numpy.random.Philox's
 * counter convention, shared by the oracle's C files.
 */
#ifndef PHILOX_ORACLE_H
#define PHILOX_ORACLE_H
#include <math.h>
#include <stdint.h>

static inline void philox4x64(const uint64_t ctr[4], const uint64_t key[2], uint64_t out[4]) {
    const uint64_t M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
    const uint64_t W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
    uint64_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const unsigned __int128 p0 = (unsigned __int128)M0 * c0;
        const unsigned __int128 p1 = (unsigned __int128)M1 * c2;
        const uint64_t hi0 = (uint64_t)(p0 >> 64), lo0 = (uint64_t)p0;
        const uint64_t hi1 = (uint64_t)(p1 >> 64), lo1 = (uint64_t)p1;
        const uint64_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static inline double u01(uint64_t x) { return (double)(x >> 11) * 0x1p-53; }

typedef struct {
    uint64_t ctr[4], key[2], buf[4];
    int pos;
} stream_t;

static inline void stream_init(stream_t *s, uint64_t c1, uint64_t c2, uint64_t c3, uint64_t k0, uint64_t k1) {
    s->ctr[0] = 0;
    s->ctr[1] = c1;
    s->ctr[2] = c2;
    s->ctr[3] = c3;
    s->key[0] = k0;
    s->key[1] = k1;
    s->pos = 4;
}

static inline double stream_uniform(stream_t *s) {
    if (s->pos == 4) {
        s->ctr[0]++;
        philox4x64(s->ctr, s->key, s->buf);
        s->pos = 0;
    }
    return u01(s->buf[s->pos++]);
}


/* Box-Muller (1958) */
static inline double box_muller(double ua, double ub) { return sqrt(-2.0 * log(1.0 - ua)) * cos(2.0 * M_PI * ub); }

#endif
