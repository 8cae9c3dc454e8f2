// Canonical 536-byte ruleset payload (crates/marl-format/src/lib.rs:70-89):
// little-endian, u8 fields one byte, f32 fields four bytes, no padding, in the
// order receptors, transport, reactions, effectors, fate, hgt_propensity,
// mutation_rate.
#include <cstring>

#include "../../include/marl_cuda.h"

namespace marl {
marl_status fail(marl_status st, const char* fmt, ...);
}

namespace {

struct Writer {
    uint8_t* p;
    void f32(float v) {
        std::memcpy(p, &v, 4);  // the host is little-endian (x86-64 / aarch64)
        p += 4;
    }
    void u8(uint8_t v) { *p++ = v; }
};

struct Reader {
    const uint8_t* p;
    float f32() {
        float v;
        std::memcpy(&v, p, 4);
        p += 4;
        return v;
    }
    uint8_t u8() { return *p++; }
};

}  // namespace

extern "C" {

marl_status marl_ruleset_pack_canonical(const marl_ruleset* rs, uint8_t out[536]) {
    if (!rs || !out) return marl::fail(MARL_ERR_INVALID_INPUT, "null argument");
    Writer w{out};
    for (const auto& r : rs->receptors) w.f32(r.k_half), w.f32(r.n_hill), w.f32(r.gain);
    for (const auto& t : rs->transport) w.f32(t.uptake_rate), w.f32(t.secrete_rate), w.u8(t.ext_species), w.u8(t.int_species);
    for (const auto& x : rs->reactions) {
        w.u8(x.substrate), w.u8(x.product), w.u8(x.catalyst), w.u8(x.cofactor);
        w.f32(x.k_m), w.f32(x.v_max), w.f32(x.k_cat);
    }
    for (const auto& e : rs->effectors) w.f32(e.threshold), w.f32(e.rate), w.u8(e.int_species), w.u8(e.ext_species);
    w.f32(rs->fate.division_energy), w.f32(rs->fate.death_energy), w.f32(rs->fate.quiescence_energy);
    w.f32(rs->fate.division_prep_ticks);
    w.f32(rs->hgt_propensity), w.f32(rs->mutation_rate);
    return (w.p - out == 536) ? MARL_OK : marl::fail(MARL_ERR_STATE, "canonical ruleset size mismatch");
}

marl_status marl_ruleset_unpack_canonical(const uint8_t in[536], marl_ruleset* rs) {
    if (!rs || !in) return marl::fail(MARL_ERR_INVALID_INPUT, "null argument");
    std::memset(rs, 0, sizeof(*rs));
    Reader r{in};
    for (auto& x : rs->receptors) x.k_half = r.f32(), x.n_hill = r.f32(), x.gain = r.f32();
    for (auto& t : rs->transport) t.uptake_rate = r.f32(), t.secrete_rate = r.f32(), t.ext_species = r.u8(), t.int_species = r.u8();
    for (auto& x : rs->reactions) {
        x.substrate = r.u8(), x.product = r.u8(), x.catalyst = r.u8(), x.cofactor = r.u8();
        x.k_m = r.f32(), x.v_max = r.f32(), x.k_cat = r.f32();
    }
    for (auto& e : rs->effectors) e.threshold = r.f32(), e.rate = r.f32(), e.int_species = r.u8(), e.ext_species = r.u8();
    rs->fate.division_energy = r.f32(), rs->fate.death_energy = r.f32(), rs->fate.quiescence_energy = r.f32();
    rs->fate.division_prep_ticks = r.f32();
    rs->hgt_propensity = r.f32(), rs->mutation_rate = r.f32();
    return MARL_OK;
}

}  // extern "C"
