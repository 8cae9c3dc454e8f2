// Seeded host RNG of the engine (seeding, division placement, mutation).
//
// The reference draws from rand 0.9.2's OS-seeded thread RNG (ChaCha12,
// crates/marl-sim/src/lib.rs:35), which has no seed and cannot be replayed.
// The engine instead uses xoshiro256** (Blackman & Vigna) seeded by four
// splitmix64 outputs, with these derived draws:
//   f32     (u64 >> 40) * 2^-24 (24 random bits, as rand's StandardUniform f32)
//   range   [lo, hi) by Lemire's multiply-and-reject on the high 32 bits
//   normal  Box-Muller in double, returned as 0.0f + std * (float)z
//           (rand_distr::Normal::sample is mean + std_dev * z)
#pragma once
#include <cmath>
#include <cstdint>

namespace marl {

class HostRng {
   public:
    explicit HostRng(uint64_t seed = 0) { seed_with(seed); }

    void seed_with(uint64_t seed) {
        uint64_t x = seed;
        for (auto& w : s_) w = mix(x);
    }
    uint64_t u64() {
        const uint64_t out = rotl(s_[1] * 5, 7) * 9;
        const uint64_t t = s_[1] << 17;
        s_[2] ^= s_[0];
        s_[3] ^= s_[1];
        s_[1] ^= s_[2];
        s_[0] ^= s_[3];
        s_[2] ^= t;
        s_[3] = rotl(s_[3], 45);
        return out;
    }
    float f32() { return (float)(u64() >> 40) * 0x1.0p-24f; }
    uint32_t range(uint32_t lo, uint32_t hi) {
        const uint32_t span = hi - lo;
        uint64_t prod = (u64() >> 32) * (uint64_t)span;
        uint32_t low = (uint32_t)prod;
        if (low < span) {
            const uint32_t reject_below = (0u - span) % span;
            while (low < reject_below) {
                prod = (u64() >> 32) * (uint64_t)span;
                low = (uint32_t)prod;
            }
        }
        return lo + (uint32_t)(prod >> 32);
    }
    float normal(float stddev) {
        const double u1 = (double)((u64() >> 11) + 1) * 0x1.0p-53;
        const double u2 = (double)(u64() >> 11) * 0x1.0p-53;
        const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
        return 0.0f + stddev * (float)z;
    }

   private:
    static uint64_t mix(uint64_t& x) {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    uint64_t s_[4];
};

}  // namespace marl
