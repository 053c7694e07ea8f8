/* rb_fill.c -- seeded synthetic input vectors for the large parity sweeps.
 *
 * TEST INFRASTRUCTURE ONLY: the tests and the benchmark use these fills to build inputs of
 * up to 2^29 elements in seconds; nothing in the product links or calls this file.
 *
 * Every element is a pure function of (distribution, seed, index): a counter-based
 * generator (the splitmix64 finaliser applied to seed and index) gives each element its own
 * random bits, so the vector is the same whatever the thread count, and a prefix of a long
 * vector is the vector of that length. The distributions follow the reference's test fills
 * (tests/common/test_util.c:1407-1600: uniform, normal, big-exponent-range and cancelling
 * fills) and the sweep's value distributions:
 *
 *   0  uniform(-1, 1)
 *   1  standard normal (Box-Muller on two uniforms of the element)
 *   2  log-uniform magnitudes 2^U(-lim, lim) with a random sign (lim 300 for double,
 *      100 for float)
 *   3  ill-conditioned: (v, -v) pairs of uniform(-1, 1) values, with 1/16 of the pairs
 *      replaced by two values of magnitude 1e-12 (random signs). Pairs are formed inside
 *      segments [0, 1024 u), [1024 u, 4096 u), [4096 u, 16384 u), ... (u = `unit` elements
 *      per item: 1 for real vectors, 2 for complex vectors, whose pairs are (z, -z)), the
 *      last segment ending at n, so every power-of-4 prefix from 1024 items is itself a set
 *      of cancelling pairs plus small values. Inside a segment of L items the item of
 *      source index j lands at position (j * A) mod L, A odd and coprime with L, which
 *      scatters each pair's two halves.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

static inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

/* random bits number `stream` of element `i` */
static inline uint64_t bits_of(uint64_t seed, uint64_t i, uint64_t stream) {
  return mix64(mix64(seed * 0x632be59bd9b4e019ull + stream) ^ (i * 0xd1b54a32d192ed03ull));
}

/* uniform in [0, 1) with 53 random bits */
static inline double u01(uint64_t b) { return (double)(b >> 11) * 0x1p-53; }

static double value_of(int dist, uint64_t seed, uint64_t i, double lim) {
  switch (dist) {
    case 0:
      return 2.0 * u01(bits_of(seed, i, 0)) - 1.0;
    case 1: {
      double u1 = 1.0 - u01(bits_of(seed, i, 1)); /* (0, 1] */
      double u2 = u01(bits_of(seed, i, 2));
      return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    }
    default: {
      uint64_t b = bits_of(seed, i, 3);
      double e = (2.0 * u01(b) - 1.0) * lim;
      double m = exp2(e);
      return (bits_of(seed, i, 4) & 1) ? -m : m;
    }
  }
}

static uint64_t gcd64(uint64_t a, uint64_t b) {
  while (b) {
    uint64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

typedef struct {
  int dist, is_float, unit;
  uint64_t seed;
  long long n, lo, hi; /* this thread's range: elements (dists 0-2) or items (dist 3) */
  void* out;
} Job;

static void put(const Job* j, long long pos, double v) {
  if (j->is_float)
    ((float*)j->out)[pos] = (float)v;
  else
    ((double*)j->out)[pos] = v;
}

/* ill-conditioned items [j->lo, j->hi) of the whole vector (items of `unit` elements) */
static void fill_illcond(const Job* j) {
  const long long items = j->n / j->unit;
  long long seg_lo = 0, seg_hi = items < 1024 ? items : 1024;
  while (seg_lo < items) {
    const long long L = seg_hi - seg_lo;
    long long a = j->lo > seg_lo ? j->lo : seg_lo;
    long long b = j->hi < seg_hi ? j->hi : seg_hi;
    if (a < b) {
      uint64_t A = 1000003ull % (uint64_t)L;
      if (A == 0) A = 1;
      while (gcd64(A, (uint64_t)L) != 1) A++;
      const long long half = L / 2;
      for (long long it = a; it < b; it++) {
        const long long src = it - seg_lo;                       /* source index in segment */
        const long long pos = seg_lo + (long long)(((uint64_t)src * A) % (uint64_t)L);
        for (int c = 0; c < j->unit; c++) {
          double v;
          if (src >= 2 * half) {
            v = 0.0; /* the odd item of an odd-length segment */
          } else {
            const long long p = src < half ? src : src - half; /* pair index */
            const uint64_t pid = (uint64_t)(seg_lo + p);
            if ((bits_of(j->seed, pid, 5) & 15) == 0) {
              v = (bits_of(j->seed, (uint64_t)(seg_lo + src) * 2 + c, 6) & 1) ? -1e-12 : 1e-12;
            } else {
              v = 2.0 * u01(bits_of(j->seed, pid * 2 + c, 7)) - 1.0;
              if (src >= half) v = -v;
            }
          }
          put(j, pos * j->unit + c, v);
        }
      }
    }
    seg_lo = seg_hi;
    seg_hi = seg_hi * 4 < items ? seg_hi * 4 : items;
  }
  /* a trailing partial item (n not a multiple of unit) */
  if (j->hi == items)
    for (long long e = items * j->unit; e < j->n; e++) put(j, e, 0.0);
}

static void* run(void* p) {
  const Job* j = (const Job*)p;
  if (j->dist == 3) {
    fill_illcond(j);
    return NULL;
  }
  const double lim = j->is_float ? 100.0 : 300.0;
  for (long long i = j->lo; i < j->hi; i++) put(j, i, value_of(j->dist, j->seed, (uint64_t)i, lim));
  return NULL;
}

static int fill(int dist, unsigned long long seed, long long n, void* out, int is_float,
                int unit, int threads) {
  if (dist < 0 || dist > 3 || n < 0 || unit < 1) return -1;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  const long long span = dist == 3 ? n / unit : n;
  pthread_t tid[256];
  int started[256] = {0};
  Job jobs[256];
  for (int t = 0; t < threads; t++) {
    jobs[t].dist = dist;
    jobs[t].is_float = is_float;
    jobs[t].unit = unit;
    jobs[t].seed = seed;
    jobs[t].n = n;
    jobs[t].lo = span * t / threads;
    jobs[t].hi = span * (t + 1) / threads;
    jobs[t].out = out;
  }
  for (int t = 1; t < threads; t++) started[t] = pthread_create(&tid[t], NULL, run, &jobs[t]) == 0;
  run(&jobs[0]);
  for (int t = 1; t < threads; t++) {
    if (started[t])
      pthread_join(tid[t], NULL);
    else
      run(&jobs[t]); /* no thread could be created: fill that range here */
  }
  return 0;
}

int rbo_fill_d(int dist, unsigned long long seed, long long n, double* out, int unit, int threads) {
  return fill(dist, seed, n, out, 0, unit, threads);
}

int rbo_fill_s(int dist, unsigned long long seed, long long n, float* out, int unit, int threads) {
  return fill(dist, seed, n, out, 1, unit, threads);
}
