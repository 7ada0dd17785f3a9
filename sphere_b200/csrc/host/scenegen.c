/*
 * scenegen.c -- native helpers of the scene builders (sphere_b200/scenes.py).
 *
 * rsa_place: random sequential placement of spheres.  Particles are placed
 * in the order given by `order` (the builders pass decreasing radius, which
 * keeps polydisperse packings near 0.3 solid fraction placeable); each draws
 * uniform positions in the box until it overlaps
 * no sphere placed before it (periodic images along x and y when requested,
 * hard floor and ceiling in z).  A cell grid of edge >= 2 r_max holds the
 * placed spheres as linked lists, so each trial tests the 27 surrounding
 * cells.  The random stream is xoshiro256** seeded by splitmix64, so a seed
 * fixes the scene on every machine.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static uint64_t sm64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct { uint64_t s[4]; } rng_t;

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t next_u64(rng_t *r)
{
    const uint64_t result = rotl(r->s[1] * 5, 7) * 9;
    const uint64_t t = r->s[1] << 17;
    r->s[2] ^= r->s[0];
    r->s[3] ^= r->s[1];
    r->s[1] ^= r->s[2];
    r->s[0] ^= r->s[3];
    r->s[2] ^= t;
    r->s[3] = rotl(r->s[3], 45);
    return result;
}

static inline double uniform01(rng_t *r) { return (double)(next_u64(r) >> 11) * 0x1.0p-53; }

/* Returns 0 on success, -1 on allocation failure, -2 when a sphere could not
 * be placed within max_trials draws (positions of placed spheres are kept). */
int rsa_place(int64_t n, const double *radii, const int64_t *order, const double L[3],
              int periodic_xy, uint64_t seed, int64_t max_trials, double *pos)
{
    double rmax = 0.0;
    for (int64_t i = 0; i < n; ++i) rmax = radii[i] > rmax ? radii[i] : rmax;
    int g[3];
    double cs[3];
    for (int d = 0; d < 3; ++d) {
        g[d] = (int)floor(L[d] / (2.0 * rmax));
        if (g[d] < 3) g[d] = 3;
        cs[d] = L[d] / g[d];
    }
    const int64_t ncell = (int64_t)g[0] * g[1] * g[2];
    int64_t *head = (int64_t *)malloc(sizeof(int64_t) * (size_t)ncell);
    int64_t *next = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    if (!head || !next) { free(head); free(next); return -1; }
    for (int64_t c = 0; c < ncell; ++c) head[c] = -1;
    rng_t rng;
    uint64_t sd = seed;
    for (int k = 0; k < 4; ++k) rng.s[k] = sm64(&sd);
    int rc = 0;
    for (int64_t k = 0; k < n && rc == 0; ++k) {
        const int64_t i = order[k];
        const double ri = radii[i];
        int64_t trial = 0;
        for (;;) {
            if (++trial > max_trials) { rc = -2; break; }
            double p[3];
            p[0] = uniform01(&rng) * L[0];
            p[1] = uniform01(&rng) * L[1];
            p[2] = ri + uniform01(&rng) * (L[2] - 2.0 * ri);
            int c[3];
            for (int d = 0; d < 3; ++d) {
                c[d] = (int)(p[d] / cs[d]);
                if (c[d] >= g[d]) c[d] = g[d] - 1;
                if (c[d] < 0) c[d] = 0;
            }
            int hit = 0;
            for (int dz = -1; dz <= 1 && !hit; ++dz) {
                const int z = c[2] + dz;
                if (z < 0 || z >= g[2]) continue;
                for (int dy = -1; dy <= 1 && !hit; ++dy) {
                    int y = c[1] + dy;
                    if (y < 0 || y >= g[1]) {
                        if (!periodic_xy) continue;
                        y = (y + g[1]) % g[1];
                    }
                    for (int dx = -1; dx <= 1 && !hit; ++dx) {
                        int x = c[0] + dx;
                        if (x < 0 || x >= g[0]) {
                            if (!periodic_xy) continue;
                            x = (x + g[0]) % g[0];
                        }
                        for (int64_t j = head[((int64_t)z * g[1] + y) * g[0] + x]; j >= 0; j = next[j]) {
                            double dd[3];
                            for (int d = 0; d < 3; ++d) dd[d] = p[d] - pos[3 * j + d];
                            if (periodic_xy) {
                                for (int d = 0; d < 2; ++d) {
                                    if (dd[d] > 0.5 * L[d]) dd[d] -= L[d];
                                    else if (dd[d] < -0.5 * L[d]) dd[d] += L[d];
                                }
                            }
                            const double rr = ri + radii[j];
                            if (dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2] < rr * rr) { hit = 1; break; }
                        }
                    }
                }
            }
            if (hit) continue;
            for (int d = 0; d < 3; ++d) pos[3 * i + d] = p[d];
            const int64_t cell = ((int64_t)c[2] * g[1] + c[1]) * g[0] + c[0];
            next[i] = head[cell];
            head[cell] = i;
            break;
        }
    }
    free(head);
    free(next);
    return rc;
}
