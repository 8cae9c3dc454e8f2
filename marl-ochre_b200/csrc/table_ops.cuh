// Warp-cooperative copies between the device cell table (structure of
// arrays, common.cuh) and a 656-byte marl_cell record, and between two table
// slots.  Lane l handles reaction l and internal species l (l < 16), the
// transporter and effector rates of slot l (l < 8), cold float l (l < 26) and
// one scalar group each (lanes 26-30).  Used by the cell-edit kernels
// (cells.cu) and by device fate processing (fate.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/marl_cuda.h"
#include "common.cuh"

namespace marl {

constexpr int kRecordU4 = (int)(sizeof(marl_cell) / 16);
static_assert(sizeof(marl_cell) % 16 == 0, "cell records are whole 16-byte words");

// Writes record `c` (shared memory, complete before the call) into table
// slot `slot` and marks its voxel in the cell map and the occupancy mask.
// The caller has checked that the position is inside the grid.
__device__ __forceinline__ void write_record_warp(const CellTable& t, const Grid g, int32_t* cmap, uint8_t* mask,
                                                  uint32_t slot, const marl_cell& c) {
    const int l = threadIdx.x & 31;
    const size_t cap = t.cap;
    const marl_ruleset& r = c.ruleset;
    if (l < MARL_R_MAX) {
        const marl_reaction& q = r.reactions[l];
        const uint32_t idx = (uint32_t)q.substrate | ((uint32_t)q.product << 8) | ((uint32_t)q.catalyst << 16) |
                             ((uint32_t)q.cofactor << 24);
        t.rx[l * cap + slot] = make_uint4(idx, __float_as_uint(q.k_m), __float_as_uint(q.v_max), __float_as_uint(q.k_cat));
        t.internal[l * cap + slot] = c.internal[l];
    }
    if (l < MARL_S_TRANSPORTERS) {
        t.tp_rate[l * cap + slot] = make_float2(r.transport[l].uptake_rate, r.transport[l].secrete_rate);
        t.ef_par[l * cap + slot] = make_float2(r.effectors[l].threshold, r.effectors[l].rate);
    }
    if (l < kColdFloats) {
        const float v = l < 3 * MARL_S_RECEPTORS
                            ? (l % 3 == 0 ? r.receptors[l / 3].k_half
                                          : (l % 3 == 1 ? r.receptors[l / 3].n_hill : r.receptors[l / 3].gain))
                            : (l == 24 ? r.hgt_propensity : r.mutation_rate);
        t.cold[(size_t)slot * kColdFloats + l] = v;
    }
    if (l == 26) {
        t.pos[slot] = pack_pos(c.pos[0], c.pos[1], c.pos[2]);
        t.age[slot] = c.age;
        const size_t row = (size_t)c.pos[2] * g.Y + c.pos[1];
        cmap[row * g.X + c.pos[0]] = (int32_t)slot;
        mask[row * mask_pitch(g.X) + c.pos[0]] = 1;
    }
    if (l == 27) {
        t.state[slot] = (uint32_t)c.prep_remaining | ((uint32_t)(c.quiescent ? 1 : 0) << 16) |
                        ((uint32_t)c.starter_type << 24);
        t.lineage[slot] = c.lineage_id;
    }
    if (l == 28 || l == 29) {
        uint32_t w[4] = {0, 0, 0, 0};
        for (int i = 0; i < 8; ++i) {
            const uint32_t pair = l == 28 ? ((uint32_t)r.transport[i].ext_species | ((uint32_t)r.transport[i].int_species << 8))
                                          : ((uint32_t)r.effectors[i].int_species | ((uint32_t)r.effectors[i].ext_species << 8));
            w[i >> 1] |= pair << ((i & 1) * 16);
        }
        (l == 28 ? t.tp_idx : t.ef_idx)[slot] = make_uint4(w[0], w[1], w[2], w[3]);
    }
    if (l == 30)
        t.fate[slot] = make_float4(r.fate.division_energy, r.fate.death_energy, r.fate.quiescence_energy,
                                   r.fate.division_prep_ticks);
}

// Reads table slot `j` into record `c` (shared memory); the caller
// synchronises the warp before using it.  Padding bytes are zeroed.
__device__ __forceinline__ void read_record_warp(const CellTable& t, uint32_t j, marl_cell& c) {
    const int l = threadIdx.x & 31;
    const size_t cap = t.cap;
    marl_ruleset& r = c.ruleset;
    if (l < MARL_R_MAX) {
        const uint4 q = t.rx[l * cap + j];
        marl_reaction& x = r.reactions[l];
        x.substrate = (uint8_t)(q.x & 0xFF);
        x.product = (uint8_t)((q.x >> 8) & 0xFF);
        x.catalyst = (uint8_t)((q.x >> 16) & 0xFF);
        x.cofactor = (uint8_t)(q.x >> 24);
        x.k_m = __uint_as_float(q.y);
        x.v_max = __uint_as_float(q.z);
        x.k_cat = __uint_as_float(q.w);
        c.internal[l] = t.internal[l * cap + j];
    }
    if (l < MARL_S_TRANSPORTERS) {
        const float2 tp = t.tp_rate[l * cap + j];
        const float2 ef = t.ef_par[l * cap + j];
        r.transport[l].uptake_rate = tp.x;
        r.transport[l].secrete_rate = tp.y;
        r.effectors[l].threshold = ef.x;
        r.effectors[l].rate = ef.y;
    }
    if (l < kColdFloats) {
        const float v = t.cold[(size_t)j * kColdFloats + l];
        if (l < 3 * MARL_S_RECEPTORS) {
            marl_receptor_params& q = r.receptors[l / 3];
            if (l % 3 == 0) q.k_half = v;
            else if (l % 3 == 1) q.n_hill = v;
            else q.gain = v;
        } else if (l == 24) {
            r.hgt_propensity = v;
        } else {
            r.mutation_rate = v;
        }
    }
    if (l == 26) {
        const uint32_t P = t.pos[j];
        c.pos[0] = (uint16_t)pos_x(P);
        c.pos[1] = (uint16_t)pos_y(P);
        c.pos[2] = (uint16_t)pos_z(P);
        c.age = t.age[j];
    }
    if (l == 27) {
        const uint32_t st = t.state[j];
        c.prep_remaining = (uint16_t)(st & 0xFFFFu);
        c.quiescent = (uint8_t)((st >> 16) & 1u);
        c.starter_type = (uint8_t)(st >> 24);
        c._pad0 = 0;
        c.lineage_id = t.lineage[j];
    }
    if (l == 28 || l == 29) {
        const uint4 q = l == 28 ? t.tp_idx[j] : t.ef_idx[j];
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
        for (int i = 0; i < 8; ++i) {
            const uint32_t pair = (w[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
            if (l == 28) {
                r.transport[i].ext_species = (uint8_t)(pair & 0xFF);
                r.transport[i].int_species = (uint8_t)(pair >> 8);
                r.transport[i]._pad[0] = r.transport[i]._pad[1] = 0;
            } else {
                r.effectors[i].int_species = (uint8_t)(pair & 0xFF);
                r.effectors[i].ext_species = (uint8_t)(pair >> 8);
                r.effectors[i]._pad[0] = r.effectors[i]._pad[1] = 0;
            }
        }
    }
    if (l == 30) {
        const float4 f = t.fate[j];
        r.fate.division_energy = f.x;
        r.fate.death_energy = f.y;
        r.fate.quiescence_energy = f.z;
        r.fate.division_prep_ticks = f.w;
    }
}

// swap_remove result (crates/marl-sim/src/lib.rs:258-267): slot d receives the
// cell in slot s and the cell map follows it.  All loads before any store.
__device__ __forceinline__ void move_one(const CellTable& t, const Grid g, int32_t* cmap, uint32_t d, uint32_t s,
                                         int l) {
    const size_t cap = t.cap;
    uint4 rx = make_uint4(0, 0, 0, 0);
    float in = 0.0f, cold = 0.0f;
    float2 tp = make_float2(0, 0), ef = make_float2(0, 0);
    if (l < MARL_R_MAX) rx = t.rx[l * cap + s], in = t.internal[l * cap + s];
    if (l < MARL_S_TRANSPORTERS) tp = t.tp_rate[l * cap + s], ef = t.ef_par[l * cap + s];
    if (l < kColdFloats) cold = t.cold[(size_t)s * kColdFloats + l];
    uint32_t pos = 0, age = 0, state = 0;
    uint64_t lineage = 0;
    uint4 w = make_uint4(0, 0, 0, 0);
    float4 fate = make_float4(0, 0, 0, 0);
    if (l == 26) pos = t.pos[s], age = t.age[s];
    if (l == 27) state = t.state[s], lineage = t.lineage[s];
    if (l == 28) w = t.tp_idx[s];
    if (l == 29) w = t.ef_idx[s];
    if (l == 30) fate = t.fate[s];
    if (l < MARL_R_MAX) t.rx[l * cap + d] = rx, t.internal[l * cap + d] = in;
    if (l < MARL_S_TRANSPORTERS) t.tp_rate[l * cap + d] = tp, t.ef_par[l * cap + d] = ef;
    if (l < kColdFloats) t.cold[(size_t)d * kColdFloats + l] = cold;
    if (l == 26) {
        t.pos[d] = pos, t.age[d] = age;
        cmap[((size_t)pos_z(pos) * g.Y + pos_y(pos)) * g.X + pos_x(pos)] = (int32_t)d;
    }
    if (l == 27) t.state[d] = state, t.lineage[d] = lineage;
    if (l == 28) t.tp_idx[d] = w;
    if (l == 29) t.ef_idx[d] = w;
    if (l == 30) t.fate[d] = fate;
}

}  // namespace marl
