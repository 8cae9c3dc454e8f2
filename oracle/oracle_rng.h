// TEST INFRASTRUCTURE ONLY — part of the CPU oracle (see oracle.cpp header).
//
// Seeded host RNG used by the oracle's seeding, division placement and
// mutation.  The reference draws from rand 0.9.2's thread-local ChaCha12,
// seeded from the OS (crates/marl-sim/src/lib.rs:35), which cannot be
// reproduced; this generator is the stand-in that the product's host engine
// also implements, so that whole runs of the oracle and of the device engine
// consume identical random streams.
//
// Specification (must stay identical to the product's host RNG):
//   state     xoshiro256** (Blackman & Vigna), 4 x u64, seeded by four
//             successive splitmix64 outputs of the 64-bit seed
//   u64       xoshiro256** output
//   f32       (u64 >> 40) * 2^-24                   — 24 random bits in [0,1)
//   range     [lo, hi) by Lemire's multiply-and-reject on (u64 >> 32)
//   normal    Box–Muller in double: u1 = ((u64>>11)+1)*2^-53, u2 = (u64>>11)*2^-53,
//             z = sqrt(-2 ln u1) * cos(2 pi u2); returns 0.0f + std * (float)z
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

struct Rng {
    uint64_t s[4];

    static uint64_t splitmix64(uint64_t& x) {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

    explicit Rng(uint64_t seed = 0) { reseed(seed); }
    void reseed(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; ++i) s[i] = splitmix64(x);
    }
    uint64_t next_u64() {
        const uint64_t result = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return result;
    }
    float next_f32() { return (float)(next_u64() >> 40) * 0x1.0p-24f; }
    // Uniform integer in [lo, hi); hi > lo.
    uint32_t range(uint32_t lo, uint32_t hi) {
        const uint32_t r = hi - lo;
        uint64_t m = (next_u64() >> 32) * (uint64_t)r;
        uint32_t l = (uint32_t)m;
        if (l < r) {
            const uint32_t t = (0u - r) % r;
            while (l < t) {
                m = (next_u64() >> 32) * (uint64_t)r;
                l = (uint32_t)m;
            }
        }
        return lo + (uint32_t)(m >> 32);
    }
    float normal(float stddev) {
        const double u1 = (double)((next_u64() >> 11) + 1) * 0x1.0p-53;
        const double u2 = (double)(next_u64() >> 11) * 0x1.0p-53;
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
        return 0.0f + stddev * (float)z;
    }
};

}  // namespace oracle

namespace oracle {

// Per-division streams of device fate processing (test infrastructure; an
// independent restatement of the product's stream specification):
//   key    = f(f(seed ^ tick*0x9E3779B97F4A7C15) ^ (parent*0xD1B54A32D192ED03 + 0x8CB92BA72F3D8DD7)),
//            f = splitmix64's finaliser
//   state  = xoshiro256** seeded by four splitmix64 outputs of key
//   u64 / f32 / range  as Rng above
//   normal Marsaglia polar: u, v = (u64>>11)*2^-52 - 1; s = u*u + v*v; retry
//          unless 0 < s < 1 (64 pairs at most, then 0); z = u*sqrt(-2 ln(s)/s);
//          0.0f + std*(float)z
//   ln(s)  frexp -> m in [0.5,1), e; m < sqrt(1/2) -> (2m, e-1);
//          t = (m-1)/(m+1); 2t * sum_{k<=10} t^(2k)/(2k+1) (Horner, fma, from
//          the top); + e*ln2 by one fma
inline uint64_t fate_finalise(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline double fate_log(double s) {
    static const double inv_odd[11] = {1.0 / 1.0,  1.0 / 3.0,  1.0 / 5.0,  1.0 / 7.0,  1.0 / 9.0, 1.0 / 11.0,
                                       1.0 / 13.0, 1.0 / 15.0, 1.0 / 17.0, 1.0 / 19.0, 1.0 / 21.0};
    int e = 0;
    double m = std::frexp(s, &e);
    if (m < std::sqrt(0.5)) {
        m *= 2.0;
        --e;
    }
    const double t = (m - 1.0) / (m + 1.0);
    const double t2 = t * t;
    double acc = inv_odd[10];
    for (int k = 9; k >= 0; --k) acc = std::fma(acc, t2, inv_odd[k]);
    const double half_log_m = t * acc;  // atanh(t)
    return std::fma((double)e, 0x1.62e42fefa39efp-1 /* ln 2 */, 2.0 * half_log_m);
}

struct FateRng : Rng {
    FateRng(uint64_t seed, uint64_t tick, uint32_t parent) : Rng(0) {
        const uint64_t a = fate_finalise(seed ^ (tick * 0x9E3779B97F4A7C15ull));
        reseed(fate_finalise(a ^ ((uint64_t)parent * 0xD1B54A32D192ED03ull + 0x8CB92BA72F3D8DD7ull)));
    }
    float normal(float stddev) {
        for (int attempt = 0; attempt < 64; ++attempt) {
            const double u = (double)(next_u64() >> 11) * 0x1.0p-52 - 1.0;
            const double v = (double)(next_u64() >> 11) * 0x1.0p-52 - 1.0;
            const double s = u * u + v * v;
            if (s > 0.0 && s < 1.0) return 0.0f + stddev * (float)(u * std::sqrt(-2.0 * fate_log(s) / s));
        }
        return 0.0f;
    }
};

}  // namespace oracle
