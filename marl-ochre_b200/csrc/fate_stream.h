// Random streams of device fate processing, and Ruleset::mutate
// (crates/marl-cell/src/cell.rs:406-524) over any generator with the engine's
// draw interface (u64, f32, range, normal).  Host and device code share it.
//
// The reference places divisions and mutates daughters with draws from one
// thread-local generator, one division after another
// (crates/marl-sim/src/lib.rs:35, :223-245), so division k's draws depend on
// every earlier division.  Device fate gives every division its own stream,
// keyed by (run seed, tick, parent index), so that divisions are placed and
// mutated in parallel with a result that does not depend on scheduling.
//
// Specification (the oracle restates it independently):
//   mix(z)   splitmix64's output function:
//            z = (z ^ z>>30) * 0xBF58476D1CE4E5B9; z = (z ^ z>>27) * 0x94D049BB133111EB; z ^ z>>31
//   key      mix(mix(seed ^ tick * 0x9E3779B97F4A7C15) ^ (parent * 0xD1B54A32D192ED03 + 0x8CB92BA72F3D8DD7))
//   state    xoshiro256** seeded with four successive splitmix64 outputs of key
//   u64 / f32 / range   as the engine's host generator: xoshiro256** output;
//            (u64 >> 40) * 2^-24; Lemire's multiply-and-reject on (u64 >> 32)
//   normal   Marsaglia's polar method (Marsaglia & Bray, 1964) in double:
//            u = (u64>>11) * 2^-52 - 1, v likewise (both exact), s = u*u + v*v
//            (two rounded products, one rounded sum); redraw both unless
//            0 < s < 1 (at most 64 pairs, then 0); z = u * sqrt(-2 ln(s) / s);
//            returns 0.0f + std * (float)z.
//   ln(s)    s = m * 2^e with m in [0.5, 1) (frexp); if m < sqrt(1/2): m *= 2,
//            e -= 1; t = (m - 1) / (m + 1); ln m = 2 t * P(t^2) with
//            P(w) = sum_{k=0..10} w^k / (2k + 1) evaluated by Horner's rule with
//            fused multiply-adds from k = 10 down (coefficients: the doubles
//            nearest 1/(2k+1)); ln s = fma(e, ln 2, ln m).  The atanh series
//            ln m = 2 atanh((m-1)/(m+1)); |t| <= 0.1716, so the truncation
//            error is below 1e-18 relative.
// Every operation is an IEEE-754 basic operation (or fma), so host and device
// produce the same bits; code that includes this header is compiled without
// floating-point contraction.
#pragma once

#include <math.h>
#include <stdint.h>

#include "../../include/marl_cuda.h"

#ifdef __CUDACC__
#define MARL_HD __host__ __device__ __forceinline__
#else
#define MARL_HD inline
#endif

namespace marl {
namespace fate {

MARL_HD uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

MARL_HD uint64_t stream_key(uint64_t seed, uint64_t tick, uint32_t parent) {
    return mix64(mix64(seed ^ (tick * 0x9E3779B97F4A7C15ull)) ^
                 ((uint64_t)parent * 0xD1B54A32D192ED03ull + 0x8CB92BA72F3D8DD7ull));
}

// Natural logarithm of s in (0, 1) by the specification above.
MARL_HD double stream_ln(double s) {
    int e = 0;
    double m = frexp(s, &e);
    if (m < 0x1.6a09e667f3bcdp-1) {
        m = m * 2.0;
        e -= 1;
    }
    const double t = (m - 1.0) / (m + 1.0);
    const double w = t * t;
    double p = 0x1.8618618618618p-5;        // 1/21
    p = fma(p, w, 0x1.af286bca1af28p-5);    // 1/19
    p = fma(p, w, 0x1.e1e1e1e1e1e1ep-5);    // 1/17
    p = fma(p, w, 0x1.1111111111111p-4);    // 1/15
    p = fma(p, w, 0x1.3b13b13b13b14p-4);    // 1/13
    p = fma(p, w, 0x1.745d1745d1746p-4);    // 1/11
    p = fma(p, w, 0x1.c71c71c71c71cp-4);    // 1/9
    p = fma(p, w, 0x1.2492492492492p-3);    // 1/7
    p = fma(p, w, 0x1.999999999999ap-3);    // 1/5
    p = fma(p, w, 0x1.5555555555555p-2);    // 1/3
    p = fma(p, w, 1.0);
    const double lnm = (2.0 * t) * p;
    return fma((double)e, 0x1.62e42fefa39efp-1, lnm);
}

// One division's stream.  `draws` counts the u64 outputs taken, so that a
// later kernel can resume the stream where an earlier one left it.
struct Stream {
    uint64_t s[4];
    uint32_t draws;

    MARL_HD explicit Stream(uint64_t key) : draws(0) {
        uint64_t x = key;
        for (int i = 0; i < 4; ++i) {
            x += 0x9E3779B97F4A7C15ull;
            s[i] = mix64(x);
        }
    }
    MARL_HD static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    MARL_HD uint64_t u64() {
        const uint64_t out = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        ++draws;
        return out;
    }
    MARL_HD void skip(uint32_t k) {
        for (uint32_t i = 0; i < k; ++i) u64();
    }
    MARL_HD float f32() { return (float)(u64() >> 40) * 0x1.0p-24f; }
    MARL_HD uint32_t range(uint32_t lo, uint32_t hi) {
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
    MARL_HD float normal(float stddev) {
        for (int tries = 0; tries < 64; ++tries) {
            const double u = (double)(u64() >> 11) * 0x1.0p-52 - 1.0;
            const double v = (double)(u64() >> 11) * 0x1.0p-52 - 1.0;
            const double uu = u * u;
            const double vv = v * v;
            const double s2 = uu + vv;
            if (s2 < 1.0 && s2 > 0.0) {
                const double z = u * sqrt(-2.0 * stream_ln(s2) / s2);
                return 0.0f + stddev * (float)z;
            }
        }
        return 0.0f;
    }
};

// Rust f32::clamp (NaN stays NaN).
MARL_HD float clamp_rs(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

template <class Rng>
MARL_HD void perturb(float& v, float rate, float sd, Rng& rng) {
    if (rng.f32() < rate) {
        v += rng.normal(sd);
        v = fmaxf(v, 0.0f);
    }
}

// Ruleset::mutate (crates/marl-cell/src/cell.rs:406-524): receptors,
// transporters (with structural species redraws), reactions (kinetics, then
// per slot a gene-duplication copy from a reaction that was active before this
// pass or a fresh species), effectors, fate thresholds, HGT propensity, and the
// meta-mutation of the mutation rate, in the reference's draw order.
template <class Rng>
MARL_HD void mutate_ruleset(marl_ruleset& rs, Rng& rng, const marl_sim_params& sim) {
    const float rate = rs.mutation_rate;
    const float sd = sim.mutation_stddev;
    const float structural = rate * sim.structural_mutation_rate_mult;
    for (int i = 0; i < MARL_S_RECEPTORS; ++i) {
        marl_receptor_params& r = rs.receptors[i];
        perturb(r.k_half, rate, sd, rng);
        perturb(r.n_hill, rate, sd, rng);
        r.n_hill = clamp_rs(r.n_hill, sim.hill_exponent_clamp_low, sim.hill_exponent_clamp_high);
        perturb(r.gain, rate, sd, rng);
    }
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) {
        marl_transport_params& t = rs.transport[i];
        perturb(t.uptake_rate, rate, sd, rng);
        perturb(t.secrete_rate, rate, sd, rng);
        if (rng.f32() < structural) t.ext_species = (uint8_t)rng.range(0, MARL_S_EXT);
        if (rng.f32() < structural) t.int_species = (uint8_t)rng.range(0, MARL_M_INT);
    }
    int donors[MARL_R_MAX];
    uint32_t n_donors = 0;
    for (int i = 0; i < MARL_R_MAX; ++i)
        if (fabsf(rs.reactions[i].v_max) > sim.active_reaction_threshold) donors[n_donors++] = i;
    for (int i = 0; i < MARL_R_MAX; ++i) {
        marl_reaction& rx = rs.reactions[i];
        perturb(rx.k_m, rate, sd, rng);
        perturb(rx.v_max, rate, sd, rng);
        perturb(rx.k_cat, rate, sd, rng);
        for (int slot = 0; slot < 3; ++slot) {
            if (rng.f32() < structural) {
                const uint32_t pick = rng.range(0, n_donors > 0 ? n_donors : 1u);
                uint8_t* dst = slot == 0 ? &rx.substrate : (slot == 1 ? &rx.product : &rx.catalyst);
                if (pick < n_donors) {
                    const int donor = donors[pick];
                    if (donor != i) {
                        const marl_reaction& d = rs.reactions[donor];
                        *dst = slot == 0 ? d.substrate : (slot == 1 ? d.product : d.catalyst);
                    }
                } else {
                    *dst = (uint8_t)rng.range(0, MARL_M_INT);
                }
            }
        }
    }
    for (int i = 0; i < MARL_S_EFFECTORS; ++i) {
        perturb(rs.effectors[i].threshold, rate, sd, rng);
        perturb(rs.effectors[i].rate, rate, sd, rng);
    }
    perturb(rs.fate.division_energy, rate, sd, rng);
    perturb(rs.fate.death_energy, rate, sd, rng);
    perturb(rs.fate.quiescence_energy, rate, sd, rng);
    perturb(rs.fate.division_prep_ticks, rate, sd, rng);
    rs.fate.division_prep_ticks = fmaxf(rs.fate.division_prep_ticks, 1.0f);
    perturb(rs.hgt_propensity, rate, sd, rng);
    if (rng.f32() < sim.meta_mutation_rate) {
        rs.mutation_rate += rng.normal(sd) * sim.meta_mutation_rate;
        rs.mutation_rate = clamp_rs(rs.mutation_rate, sim.meta_mutation_clamp_low, sim.meta_mutation_clamp_high);
    }
}

}  // namespace fate
}  // namespace marl
