// Host side of one run's tick loop: the parts of marl_sim::run that stay on
// the host (crates/marl-sim/src/lib.rs:34-105 seeding, :219-277 fate
// processing), shared by the single-run engine and the batch.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/marl_cuda.h"
#include "host_rng.h"

namespace marl {

// What the host keeps per cell: the data the device never changes during a
// tick (position, lineage, starter type, ruleset).
struct HostCell {
    uint16_t pos[3];
    uint8_t starter_type;
    uint64_t lineage_id;
    marl_ruleset ruleset;
};

// The result of one tick's fate processing, ready for marl_apply_edits.
struct EditData {
    std::vector<uint32_t> halve, deaths, move_dst, move_src;
    uint32_t n_after_deaths = 0;
    std::vector<marl_cell> births;
    marl_edit_list view() const;
};

class HostRun {
   public:
    int X = 0, Y = 0, Z = 0;
    marl_sim_params sim{};
    HostRng rng;
    uint64_t seed = 0;            // rng_seed of the run (also keys device fate streams)
    std::vector<HostCell> cells;  // the reference's `cells: Vec<CellState>` order
    std::vector<int32_t> cmap;    // the reference's `cell_map` as a dense voxel map
    uint64_t tick = 0, total_div = 0, total_death = 0, tick_div = 0, tick_death = 0;

    void init(int gx, int gy, int gz, const marl_sim_params& p, uint64_t seed);
    // init_field_boundaries + seed_cells x3 (seeding.rs:9-58, lib.rs:59-105):
    // fills `field` ([z][y][x][12]) and returns the seeded cells.
    marl_status seed_default(uint32_t seed_count, std::vector<float>& field, std::vector<marl_cell>& out);
    // Takes over an existing cell vector (positions assumed valid and unique).
    void adopt(const marl_cell* c, uint32_t n);
    // Fate processing of one tick's ordered change list (lib.rs:219-277).
    marl_status process(const marl_change* changes, uint32_t count, EditData& out);

   private:
    size_t vox(int x, int y, int z) const { return ((size_t)z * Y + y) * X + x; }
    bool find_empty_neighbor(const uint16_t p[3], uint16_t out[3]);
};

}  // namespace marl
