// Host engine: the tick loop of marl_sim::run (crates/marl-sim/src/lib.rs:34-277)
// over a device context.  Each tick the device runs sources, diffusion, light
// and the cell loop and returns the ordered change list of Division/Death
// events; the host then performs the reference's fate processing — division
// placement, cloning, halving, mutation, lineage draws, swap_remove deaths and
// appended births — with its seeded RNG, and sends the resulting edit list
// back.  File output (dumps, CSV, images) is not part of this path.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/marl_cuda.h"
#include "engine_host.h"
#include "fate_stream.h"
#include "host_rng.h"

namespace marl {
marl_status fail(marl_status st, const char* fmt, ...);
}
using marl::EditData;
using marl::fail;
using marl::HostCell;
using marl::HostRng;
using marl::HostRun;

namespace {

// crates/marl-sim/src/spatial.rs:8-15
const int kFace[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// ---- starter metabolisms (crates/marl-sim/src/starter_metabolisms.rs) ----
void set_inactive(marl_ruleset& r) {  // :6-42
    std::memset(&r, 0, sizeof(r));
    for (auto& x : r.receptors) x = marl_receptor_params{1.0f, 2.0f, 0.0f};
    for (auto& x : r.transport) x = marl_transport_params{0.0f, 0.0f, 0, 0, {0, 0}};
    for (auto& x : r.reactions) x = marl_reaction{0, 0, 0, MARL_NO_COFACTOR, 1.0f, 0.0f, 0.5f};
    for (auto& x : r.effectors) x = marl_effector_params{10.0f, 0.0f, 0, 0, {0, 0}};
}

marl_cell starter(int kind, const uint16_t pos[3], uint64_t lineage) {
    marl_cell c;
    std::memset(&c, 0, sizeof(c));
    std::memcpy(c.pos, pos, sizeof(c.pos));
    c.lineage_id = lineage;
    c.starter_type = (uint8_t)kind;
    marl_ruleset& r = c.ruleset;
    set_inactive(r);
    r.hgt_propensity = 0.1f;
    r.mutation_rate = 0.05f;
    const uint8_t N = MARL_NO_COFACTOR;
    if (kind == 0) {  // phototroph, :46-187
        r.receptors[2] = {0.3f, 2.0f, 1.0f};
        r.receptors[3] = {0.5f, 2.0f, 1.0f};
        r.transport[0] = {0.6f, 0.0f, 3, 3, {0, 0}};
        r.transport[1] = {0.0f, 0.6f, 1, 1, {0, 0}};
        r.transport[2] = {0.0f, 0.3f, 4, 4, {0, 0}};
        r.transport[3] = {0.1f, 0.0f, 2, 2, {0, 0}};
        r.reactions[0] = {3, 0, 15, N, 0.2f, 0.8f, 0.1f};
        r.reactions[1] = {3, 1, 15, N, 0.2f, 0.4f, 0.1f};
        r.reactions[2] = {3, 4, 0, N, 0.3f, 0.3f, 0.3f};
        r.reactions[3] = {3, 5, 6, N, 0.3f, 0.15f, 0.1f};
        r.reactions[4] = {3, 6, 5, N, 0.3f, 0.1f, 0.1f};
        r.effectors[0] = {0.5f, 0.8f, 1, 1, {0, 0}};
        r.effectors[1] = {1.0f, 0.2f, 4, 4, {0, 0}};
        r.fate = {1.2f, 0.05f, 0.15f, 20.0f};
        c.internal[0] = 0.3f, c.internal[3] = 0.3f, c.internal[5] = 0.05f, c.internal[6] = 0.05f;
    } else if (kind == 1) {  // chemolithotroph, :191-326
        r.receptors[1] = {0.3f, 2.0f, 1.0f};
        r.receptors[2] = {0.3f, 2.0f, 1.0f};
        r.transport[0] = {0.7f, 0.0f, 1, 1, {0, 0}};
        r.transport[1] = {0.7f, 0.0f, 2, 2, {0, 0}};
        r.transport[2] = {0.2f, 0.0f, 3, 3, {0, 0}};
        r.transport[3] = {0.0f, 0.3f, 4, 4, {0, 0}};
        r.reactions[0] = {2, 0, 5, 1, 0.15f, 0.7f, 0.1f};
        r.reactions[1] = {1, 4, 0, N, 0.3f, 0.3f, 0.2f};
        r.reactions[2] = {7, 0, 5, N, 0.3f, 0.15f, 0.1f};
        r.reactions[3] = {3, 5, 6, N, 0.3f, 0.15f, 0.1f};
        r.reactions[4] = {3, 6, 5, N, 0.3f, 0.1f, 0.1f};
        r.effectors[0] = {0.5f, 0.3f, 4, 4, {0, 0}};
        r.fate = {1.0f, 0.05f, 0.12f, 20.0f};
        c.internal[0] = 1.5f, c.internal[1] = 0.5f, c.internal[2] = 0.5f;
        c.internal[5] = 0.05f, c.internal[6] = 0.05f, c.internal[7] = 5.0f;
    } else {  // anaerobe, :330-459
        r.receptors[2] = {0.3f, 2.0f, 1.0f};
        r.transport[0] = {0.9f, 0.0f, 2, 2, {0, 0}};
        r.transport[1] = {0.3f, 0.0f, 3, 3, {0, 0}};
        r.transport[2] = {0.0f, 0.5f, 4, 4, {0, 0}};
        r.transport[3] = {0.1f, 0.0f, 1, 1, {0, 0}};
        r.reactions[0] = {2, 0, 5, N, 0.15f, 0.8f, 0.1f};
        r.reactions[1] = {3, 4, 0, N, 0.2f, 0.3f, 0.2f};
        r.reactions[2] = {0, 3, 1, N, 0.01f, 2.0f, 0.01f};
        r.reactions[3] = {3, 5, 6, N, 0.3f, 0.15f, 0.1f};
        r.reactions[4] = {3, 6, 5, N, 0.3f, 0.1f, 0.1f};
        r.effectors[0] = {0.5f, 0.5f, 4, 4, {0, 0}};
        r.fate = {0.8f, 0.05f, 0.1f, 20.0f};
        c.internal[0] = 0.5f, c.internal[2] = 0.7f, c.internal[5] = 0.05f, c.internal[6] = 0.05f;
    }
    return c;
}

}  // namespace

namespace marl {

marl_edit_list EditData::view() const {
    marl_edit_list e;
    e.n_halve = (uint32_t)halve.size();
    e.halve = halve.data();
    e.n_deaths = (uint32_t)deaths.size();
    e.deaths = deaths.data();
    e.n_moves = (uint32_t)move_dst.size();
    e.move_dst = move_dst.data();
    e.move_src = move_src.data();
    e.n_after_deaths = n_after_deaths;
    e.n_births = (uint32_t)births.size();
    e.births = births.data();
    return e;
}

void HostRun::init(int gx, int gy, int gz, const marl_sim_params& p, uint64_t seed) {
    X = gx, Y = gy, Z = gz;
    sim = p;
    this->seed = seed;
    rng.seed_with(seed);
    cells.clear();
    cmap.assign((size_t)gx * gy * gz, -1);
    tick = total_div = total_death = tick_div = tick_death = 0;
}

marl_status HostRun::seed_default(uint32_t seed_count, std::vector<float>& field, std::vector<marl_cell>& out) {
    if (X <= 2 * (int)sim.seed_margin || Y <= 2 * (int)sim.seed_margin)
        return fail(MARL_ERR_INVALID_INPUT, "grid %dx%d too small for seed_margin %u", X, Y, sim.seed_margin);
    // init_field_boundaries (crates/marl-sim/src/seeding.rs:9-26)
    field.assign((size_t)X * Y * Z * MARL_S_EXT, 0.0f);
    const int layers = (int)sim.boundary_prime_layers;
    for (int y = 0; y < Y; ++y)
        for (int x = 0; x < X; ++x) {
            for (int z = 0; z < layers && z < Z; ++z) {
                field[vox(x, y, z) * 12 + 1] = sim.boundary_prime_oxidant;
                field[vox(x, y, z) * 12 + 3] = sim.boundary_prime_carbon;
            }
            for (int z = std::max(Z - layers, 0); z < Z; ++z) field[vox(x, y, z) * 12 + 2] = sim.boundary_prime_reductant;
        }
    // seed_cells x3 with depth bands scaled by Z/200 (lib.rs:59-105, seeding.rs:28-58)
    out.clear();
    const float z_scale = (float)Z / 200.0f;
    const float lo_f[3] = {sim.phototroph_z_lo, sim.chemolithotroph_z_lo, sim.anaerobe_z_lo};
    const float hi_f[3] = {sim.phototroph_z_hi, sim.chemolithotroph_z_hi, sim.anaerobe_z_hi};
    const float min_span[3] = {1.0f, 3.0f, 3.0f};
    for (int kind = 0; kind < 3; ++kind) {
        const uint16_t lo = (uint16_t)(lo_f[kind] * z_scale);
        const uint16_t hi = (uint16_t)std::fmax(hi_f[kind] * z_scale, (float)lo + min_span[kind]);
        const uint32_t zhi = std::min<uint32_t>(hi, (uint32_t)Z);
        if (seed_count > 0 && lo >= zhi) return fail(MARL_ERR_INVALID_INPUT, "empty seeding depth band [%u,%u)", lo, zhi);
        uint32_t seeded = 0;
        for (uint32_t a = 0; a < seed_count * 8 && seeded < seed_count; ++a) {
            const uint16_t x = (uint16_t)rng.range(sim.seed_margin, (uint32_t)X - sim.seed_margin);
            const uint16_t y = (uint16_t)rng.range(sim.seed_margin, (uint32_t)Y - sim.seed_margin);
            const uint16_t z = (uint16_t)rng.range(lo, zhi);
            const size_t v = vox(x, y, z);
            if (cmap[v] >= 0) continue;
            const uint16_t pos[3] = {x, y, z};
            const marl_cell c = starter(kind, pos, rng.u64());
            cmap[v] = (int32_t)out.size();
            out.push_back(c);
            ++seeded;
        }
    }
    adopt(out.data(), (uint32_t)out.size());
    return MARL_OK;
}

void HostRun::adopt(const marl_cell* c, uint32_t n) {
    cells.clear();
    std::fill(cmap.begin(), cmap.end(), -1);
    for (uint32_t i = 0; i < n; ++i) {
        HostCell h;
        std::memcpy(h.pos, c[i].pos, sizeof(h.pos));
        h.starter_type = c[i].starter_type;
        h.lineage_id = c[i].lineage_id;
        h.ruleset = c[i].ruleset;
        cells.push_back(h);
        cmap[vox(h.pos[0], h.pos[1], h.pos[2])] = (int32_t)i;
    }
}

// crates/marl-sim/src/spatial.rs:115-154 (find_empty_neighbor)
bool HostRun::find_empty_neighbor(const uint16_t p[3], uint16_t out[3]) {
    const int dist = (int)sim.division_neighbor_distance;
    uint16_t cand[6][3];
    uint32_t nc = 0;
    for (const auto& f : kFace) {
        const int nx = p[0] + f[0] * dist, ny = p[1] + f[1] * dist, nz = p[2] + f[2] * dist;
        if (nx >= 0 && nx < X && ny >= 0 && ny < Y && nz >= 0 && nz < Z && cmap[vox(nx, ny, nz)] < 0) {
            cand[nc][0] = (uint16_t)nx, cand[nc][1] = (uint16_t)ny, cand[nc][2] = (uint16_t)nz;
            ++nc;
        }
    }
    if (nc == 0) {
        for (const auto& f : kFace) {
            const int nx = p[0] + f[0], ny = p[1] + f[1], nz = p[2] + f[2];
            if (nx >= 0 && nx < X && ny >= 0 && ny < Y && nz >= 0 && nz < Z && cmap[vox(nx, ny, nz)] < 0) {
                cand[nc][0] = (uint16_t)nx, cand[nc][1] = (uint16_t)ny, cand[nc][2] = (uint16_t)nz;
                ++nc;
            }
        }
        if (nc == 0) return false;
    }
    const uint32_t i = rng.range(0, nc);
    std::memcpy(out, cand[i], sizeof(uint16_t) * 3);
    return true;
}

// crates/marl-sim/src/lib.rs:219-277 (fate processing) -> edit list.
//
// The reference's order of events and of random draws is kept exactly; what
// differs is only how the memory is walked.  The cell rows and cell-map
// entries that the step will touch sit at random places in tens of megabytes,
// so a first pass over the change list prefetches them all (the misses then
// overlap instead of following one another), daughters are built in place in
// the edit list, and the swap_remove bookkeeping keeps an entry per death
// instead of one per cell.
marl_status HostRun::process(const marl_change* changes, uint32_t count, EditData& e) {
    tick_div = tick_death = 0;
    e.halve.clear(), e.deaths.clear(), e.move_dst.clear(), e.move_src.clear(), e.births.clear();
    const uint32_t n0 = (uint32_t)cells.size();
    uint32_t n_div = 0;
    for (uint32_t k = 0; k < count; ++k) {
        if (changes[k].cell >= n0)
            return fail(MARL_ERR_STATE, "change list names cell %u of %u", changes[k].cell, n0);
        n_div += changes[k].event == MARL_EVENT_DIVISION;
    }
    // Prefetch: parents' rows and every cell-map entry a placement may probe,
    // dying cells' rows and voxels.
    const int dist = (int)sim.division_neighbor_distance;
    for (uint32_t k = 0; k < count; ++k) {
        const marl_change& ch = changes[k];
        if (ch.event != MARL_EVENT_DIVISION && ch.event != MARL_EVENT_DEATH) continue;
        const HostCell& c = cells[ch.cell];
        const char* row = reinterpret_cast<const char*>(&c);
        for (size_t o = 0; o < sizeof(HostCell); o += 64) __builtin_prefetch(row + o);
        for (const auto& f : kFace)
            for (int d : {dist, 1}) {
                const int nx = c.pos[0] + f[0] * d, ny = c.pos[1] + f[1] * d, nz = c.pos[2] + f[2] * d;
                if (nx >= 0 && nx < X && ny >= 0 && ny < Y && nz >= 0 && nz < Z) __builtin_prefetch(&cmap[vox(nx, ny, nz)]);
            }
    }
    e.births.reserve(n_div);
    for (uint32_t k = 0; k < count; ++k) {
        const marl_change& ch = changes[k];
        if (ch.event == MARL_EVENT_DIVISION) {
            const HostCell& parent = cells[ch.cell];
            uint16_t dpos[3];
            if (find_empty_neighbor(parent.pos, dpos)) {
                e.births.emplace_back();
                marl_cell& d = e.births.back();
                std::memset(&d, 0, sizeof(d));
                std::memcpy(d.pos, dpos, sizeof(dpos));
                d.quiescent = ch.quiescent;
                d.starter_type = parent.starter_type;
                d.age = 0;
                d.prep_remaining = 0;
                d.lineage_id = rng.u64();
                for (int i = 0; i < MARL_M_INT; ++i) d.internal[i] = ch.internal[i] * 0.5f;
                d.ruleset = parent.ruleset;
                e.halve.push_back(ch.cell);
                marl::fate::mutate_ruleset(d.ruleset, rng, sim);  // cell.rs:406-524
                ++tick_div;
            }
        } else if (ch.event == MARL_EVENT_DEATH) {
            e.deaths.push_back(ch.cell);
            ++tick_death;
        }
    }
    total_div += tick_div;
    total_death += tick_death;
    // Deaths arrive in ascending cell order without duplicates (one event per
    // cell); remove them back to front with swap_remove.  Only death slots
    // ever receive another cell, so the original slot of the cell in slot i is
    // recorded per death (origin_of(i) = i for every other slot).
    const std::vector<uint32_t>& D = e.deaths;
    std::vector<uint32_t> org(D.size());
    std::vector<uint8_t> has(D.size(), 0);
    auto origin_of = [&](uint32_t i) -> uint32_t {
        const auto it = std::lower_bound(D.begin(), D.end(), i);
        if (it == D.end() || *it != i) return i;
        const size_t k = (size_t)(it - D.begin());
        return has[k] ? org[k] : i;
    };
    for (size_t k = D.size(); k-- > 0;) {
        const uint32_t i = D[k];
        const uint32_t last = (uint32_t)cells.size() - 1;
        cmap[vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = -1;
        const uint32_t o = origin_of(last);
        if (i != last) cells[i] = cells[last];
        org[k] = o;
        has[k] = 1;
        cells.pop_back();
        if (i < cells.size()) cmap[vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = (int32_t)i;
    }
    e.n_after_deaths = (uint32_t)cells.size();
    for (size_t k = 0; k < D.size(); ++k)
        if (D[k] < e.n_after_deaths && org[k] != D[k]) {
            e.move_dst.push_back(D[k]);
            e.move_src.push_back(org[k]);
        }
    // Births append unless the voxel was taken meanwhile (lib.rs:270-277);
    // rejected daughters leave the edit list, the others keep their order.
    size_t w = 0;
    for (size_t r = 0; r < e.births.size(); ++r) {
        const marl_cell& b = e.births[r];
        const size_t v = vox(b.pos[0], b.pos[1], b.pos[2]);
        if (cmap[v] >= 0) continue;
        cmap[v] = (int32_t)cells.size();
        cells.emplace_back();
        HostCell& h = cells.back();
        std::memcpy(h.pos, b.pos, sizeof(h.pos));
        h.starter_type = b.starter_type;
        h.lineage_id = b.lineage_id;
        h.ruleset = b.ruleset;
        if (w != r) e.births[w] = b;
        ++w;
    }
    e.births.resize(w);
    ++tick;
    return MARL_OK;
}

}  // namespace marl

struct marl_engine {
    marl_ctx* ctx = nullptr;
    HostRun run;
    bool device_fate = false;  // fate on the device (marl_engine_set_device_fate)
    uint64_t population = 0;   // device fate: population after the last step
    EditData edits;
    std::vector<marl_change> changes;
    uint64_t h2d_last = 0, d2h_last = 0;

    marl_status step_once() {
        uint32_t count = 0;
        if (changes.size() < run.cells.size() + 1) changes.resize(run.cells.size() + 1);
        marl_status st = marl_tick(ctx, changes.data(), (uint32_t)changes.size(), &count);
        if (st) return st;
        if ((st = run.process(changes.data(), count, edits))) return st;
        const marl_edit_list e = edits.view();
        return marl_apply_edits(ctx, &e);
    }
};

extern "C" {

// Transfer counters are read from the context.
uint64_t marl_internal_ctx_h2d(marl_ctx* c);
uint64_t marl_internal_ctx_d2h(marl_ctx* c);

marl_status marl_engine_create(int32_t gx, int32_t gy, int32_t gz, const marl_sim_params* sim, uint64_t rng_seed,
                               uint32_t seed_count, uint32_t cell_capacity, marl_engine** out) {
    if (!sim || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *out = nullptr;
    marl_engine* e = new (std::nothrow) marl_engine();
    if (!e) return fail(MARL_ERR_OUT_OF_MEMORY, "host allocation");
    e->run.init(gx, gy, gz, *sim, rng_seed);
    std::vector<float> field;
    std::vector<marl_cell> cells;
    marl_status st = e->run.seed_default(seed_count, field, cells);
    if (!st && cells.size() > cell_capacity)
        st = fail(MARL_ERR_CAPACITY, "%zu seeded cells exceed capacity %u", cells.size(), cell_capacity);
    if (!st) st = marl_ctx_create(gx, gy, gz, sim, cell_capacity, &e->ctx);
    if (!st) st = marl_upload_field(e->ctx, field.data());
    if (!st) st = marl_upload_cells(e->ctx, cells.data(), (uint32_t)cells.size());
    if (st) {
        marl_engine_destroy(e);
        return st;
    }
    *out = e;
    return MARL_OK;
}

marl_status marl_engine_create_from_state(int32_t gx, int32_t gy, int32_t gz, const marl_sim_params* sim,
                                          uint64_t rng_seed, const float* field, const marl_cell* cells, uint32_t n,
                                          uint32_t cell_capacity, marl_engine** out) {
    if (!sim || !out || !field || (n && !cells)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *out = nullptr;
    marl_engine* e = new (std::nothrow) marl_engine();
    if (!e) return fail(MARL_ERR_OUT_OF_MEMORY, "host allocation");
    marl_status st = marl_ctx_create(gx, gy, gz, sim, cell_capacity, &e->ctx);
    if (!st) st = marl_upload_field(e->ctx, field);
    if (!st) st = marl_upload_cells(e->ctx, cells, n);  // validates positions
    if (st) {
        marl_engine_destroy(e);
        return st;
    }
    e->run.init(gx, gy, gz, *sim, rng_seed);
    e->run.adopt(cells, n);
    *out = e;
    return MARL_OK;
}

void marl_engine_destroy(marl_engine* e) {
    if (!e) return;
    if (e->ctx) marl_ctx_destroy(e->ctx);
    delete e;
}

marl_status marl_engine_set_stream(marl_engine* e, void* stream) {
    if (!e) return fail(MARL_ERR_INVALID_INPUT, "null engine");
    return marl_ctx_set_stream(e->ctx, stream);
}

marl_status marl_engine_step(marl_engine* e, uint32_t ticks) {
    if (!e) return fail(MARL_ERR_INVALID_INPUT, "null engine");
    if (e->device_fate) {
        const uint64_t h0 = marl_internal_ctx_h2d(e->ctx), d0 = marl_internal_ctx_d2h(e->ctx);
        marl_status st = marl_ctx_run_ticks(e->ctx, ticks);
        if (st) return st;
        marl_fate_stats fs;
        if ((st = marl_ctx_fate_stats(e->ctx, &fs))) return st;
        e->run.tick = fs.tick;
        e->run.total_div = fs.total_divisions;
        e->run.total_death = fs.total_deaths;
        e->run.tick_div = fs.tick_divisions;
        e->run.tick_death = fs.tick_deaths;
        e->population = fs.population;
        const uint64_t t = ticks ? ticks : 1;
        e->h2d_last = (marl_internal_ctx_h2d(e->ctx) - h0) / t;
        e->d2h_last = (marl_internal_ctx_d2h(e->ctx) - d0) / t;
        return MARL_OK;
    }
    for (uint32_t t = 0; t < ticks; ++t) {
        const uint64_t h0 = marl_internal_ctx_h2d(e->ctx), d0 = marl_internal_ctx_d2h(e->ctx);
        marl_status st = e->step_once();
        if (st) return st;
        e->h2d_last = marl_internal_ctx_h2d(e->ctx) - h0;
        e->d2h_last = marl_internal_ctx_d2h(e->ctx) - d0;
    }
    return MARL_OK;
}

marl_status marl_engine_stats_get(marl_engine* e, marl_engine_stats* s) {
    if (!e || !s) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    s->tick = e->run.tick;
    s->population = e->device_fate ? e->population : e->run.cells.size();
    s->total_divisions = e->run.total_div;
    s->total_deaths = e->run.total_death;
    s->tick_divisions = e->run.tick_div;
    s->tick_deaths = e->run.tick_death;
    s->h2d_bytes_last_tick = e->h2d_last;
    s->d2h_bytes_last_tick = e->d2h_last;
    return MARL_OK;
}

marl_status marl_engine_get_cells(marl_engine* e, marl_cell* out, uint32_t cap, uint32_t* n_out) {
    if (!e) return fail(MARL_ERR_INVALID_INPUT, "null engine");
    return marl_download_cells(e->ctx, out, cap, n_out);
}

marl_status marl_engine_get_field(marl_engine* e, float* field) {
    if (!e) return fail(MARL_ERR_INVALID_INPUT, "null engine");
    return marl_download_field(e->ctx, field);
}

marl_status marl_engine_get_light(marl_engine* e, float* light) {
    if (!e) return fail(MARL_ERR_INVALID_INPUT, "null engine");
    return marl_download_light(e->ctx, light);
}

marl_ctx* marl_engine_ctx(marl_engine* e) { return e ? e->ctx : nullptr; }

marl_status marl_engine_set_device_fate(marl_engine* e, int32_t enable) {
    if (!e) return fail(MARL_ERR_INVALID_INPUT, "null engine");
    const bool on = enable != 0;
    if (on == e->device_fate) return MARL_OK;
    marl_status st;
    if (on) {
        if ((st = marl_ctx_fate_init(e->ctx, e->run.seed, e->run.tick, e->run.total_div, e->run.total_death)))
            return st;
        e->population = e->run.cells.size();
        e->device_fate = true;
        return MARL_OK;
    }
    // Back to host fate: the host takes over the device's cell vector (its
    // sequential stream continues where it stood).
    uint32_t n = 0;
    if ((st = marl_download_cells(e->ctx, nullptr, 0, &n))) return st;
    std::vector<marl_cell> cells(n);
    if (n && (st = marl_download_cells(e->ctx, cells.data(), n, &n))) return st;
    e->run.adopt(cells.data(), n);
    e->device_fate = false;
    return MARL_OK;
}

}  // extern "C"
