// Seeded synthetic input generator (see include/gcz_gen.h for the model).
#include "gcz_gen.h"

#include <cmath>
#include <cstring>

namespace {

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t &x) {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto &v : s) v = splitmix(x);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256**
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in (0, 1]
    double unit() { return ((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
};

// Geometric number of failures before the first success, mean m (m >= 0).
uint64_t geometric0(Rng &r, double m) {
    if (m <= 0.0) return 0;
    const double q = m / (m + 1.0);  // continue probability
    return (uint64_t)std::floor(std::log(r.unit()) / std::log(q));
}

constexpr double kSpanMean = 48.0;
constexpr int kAlpha = 64;
constexpr int kRowQ = 1024;

}  // namespace

extern "C" void gcz_gen_synthetic(uint64_t seed, uint8_t *out, uint64_t n, uint64_t max_offset,
                                  double f_markov, double f_copy, double f_random) {
    if (!out || n == 0) return;
    double tot = f_markov + f_copy + f_random;
    if (!(tot > 0.0)) {
        f_markov = 0.4;
        f_copy = 0.4;
        f_random = 0.2;
        tot = 1.0;
    }
    const double p_markov = f_markov / tot, p_copy = p_markov + f_copy / tot;
    if (max_offset < 1) max_offset = 1;
    Rng rng(seed);

    // Alphabet: a seeded choice of 64 distinct byte values.
    uint8_t perm[256];
    for (int i = 0; i < 256; i++) perm[i] = (uint8_t)i;
    for (int i = 255; i > 0; i--) {
        int j = (int)(rng.next() % (uint64_t)(i + 1));
        uint8_t t = perm[i];
        perm[i] = perm[j];
        perm[j] = t;
    }
    uint8_t alpha[kAlpha];
    std::memcpy(alpha, perm, kAlpha);

    // Transition rows: Zipf(1) over a seeded permutation, quantised to kRowQ slots.
    static thread_local uint8_t row[kAlpha][kRowQ];
    double w[kAlpha], wsum = 0.0;
    for (int k = 0; k < kAlpha; k++) wsum += (w[k] = 1.0 / (k + 1));
    for (int s = 0; s < kAlpha; s++) {
        int order[kAlpha];
        for (int k = 0; k < kAlpha; k++) order[k] = k;
        for (int k = kAlpha - 1; k > 0; k--) {
            int j = (int)(rng.next() % (uint64_t)(k + 1));
            int t = order[k];
            order[k] = order[j];
            order[j] = t;
        }
        int fill = 0;
        for (int k = 0; k < kAlpha && fill < kRowQ; k++) {
            int cnt = (int)std::floor(w[k] / wsum * kRowQ + 0.5);
            for (int c = 0; c < cnt && fill < kRowQ; c++) row[s][fill++] = (uint8_t)order[k];
        }
        while (fill < kRowQ) row[s][fill++] = (uint8_t)order[0];  // rounding remainder
    }

    const double log_max = std::log((double)max_offset + 1.0);
    uint64_t pos = 0;
    int state = (int)(rng.next() % kAlpha);
    while (pos < n) {
        const double u = rng.unit();
        int kind = u <= p_markov ? 0 : (u <= p_copy ? 1 : 2);
        if (kind == 1 && pos == 0) kind = 0;
        if (kind == 1) {
            uint64_t len = 4 + geometric0(rng, kSpanMean - 4.0);
            uint64_t off = (uint64_t)std::floor(std::exp(rng.unit() * log_max));
            if (off < 1) off = 1;
            if (off > max_offset) off = max_offset;
            if (off > pos) off = pos;
            if (len > n - pos) len = n - pos;
            const uint8_t *from = out + pos - off;
            for (uint64_t i = 0; i < len; i++) out[pos + i] = from[i];  // overlapping copies repeat
            pos += len;
        } else {
            uint64_t len = 1 + geometric0(rng, kSpanMean - 1.0);
            if (len > n - pos) len = n - pos;
            if (kind == 0) {
                for (uint64_t i = 0; i < len; i++) {
                    state = row[state][rng.next() & (kRowQ - 1)];
                    out[pos + i] = alpha[state];
                }
            } else {
                uint64_t i = 0;
                while (i < len) {
                    uint64_t r = rng.next();
                    for (int b = 0; b < 8 && i < len; b++, i++) out[pos + i] = (uint8_t)(r >> (8 * b));
                }
            }
            pos += len;
        }
    }
}

extern "C" void gcz_gen_file_sizes(uint64_t seed, uint64_t count, uint64_t min_size, uint64_t max_size,
                                   uint64_t *sizes, double *mix) {
    if (!sizes) return;
    if (min_size < 1) min_size = 1;
    if (max_size < min_size) max_size = min_size;
    Rng rng(seed ^ 0x5EEDF11E5ull);
    const double lo = std::log((double)min_size), hi = std::log((double)max_size);
    for (uint64_t i = 0; i < count; i++) {
        double s = std::exp(lo + (hi - lo) * (1.0 - rng.unit()));
        uint64_t v = (uint64_t)s;
        if (v < min_size) v = min_size;
        if (v > max_size) v = max_size;
        sizes[i] = v;
        double e0 = -std::log(rng.unit()), e1 = -std::log(rng.unit()), e2 = -std::log(rng.unit());
        double t = e0 + e1 + e2;
        if (mix) {
            mix[3 * i + 0] = e0 / t;
            mix[3 * i + 1] = e1 / t;
            mix[3 * i + 2] = e2 / t;
        }
    }
}
