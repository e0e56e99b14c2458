// worklist.cuh -- persistent passes over a device work list of many items.
//
// An uneven batch (polynomials of different sizes, BabyBear and M31 mixed)
// runs each phase of its LDEs -- the inverse low layers, the expansion, the
// forward low layers -- as ONE persistent launch for every item at once,
// instead of one launch per item and phase.  The work list lives in global
// memory:
//   * WorkItem: one item's pass -- its two tensor maps (input, output), its
//     pass arguments (twiddles, sizes, columns), its field and layer count;
//   * WorkUnit: (item, first tile, end tile), a run of consecutive tiles of
//     one item.
// Every CTA pops units with an atomic counter (thread 0 pops, the tile ids
// reach the other threads through shared memory), keeps the next tile's TMA
// load in flight while it computes the current one -- across unit and item
// boundaries -- and runs each tile with the tile engine of its field and
// layer count (TPass::tile_body: the same rounds, twiddles and exchanges as
// the single-item passes, so results are bit-identical).
#pragma once
#include <cstdint>
#include <vector>

#include "context.hpp"
#include "tile_tma.cuh"

namespace sfntt {

struct alignas(128) WorkItem {
  CUtensorMap min;   // input map (tiles of 2^13 words, the pass's own shape)
  CUtensorMap mout;  // output map
  TmaArgs a;         // the pass's arguments (as the single-item launch sets them)
  int32_t field;     // SFNTT_BABYBEAR or SFNTT_M31
  int32_t P;         // contiguous passes: layers 5..13; expansions: 8
  uint32_t lstage;   // expansions: BabyBear twiddle chunks staged in shared memory
  uint32_t pad;
};

struct WorkUnit {
  uint32_t item, t0, t1;  // tiles [t0, t1) of work item `item`
};

// Work-list counters: one per phase, zeroed before the phase's launch.
constexpr int kWorkPhases = 3;

// Host side of one phase: its items and units (copied to the device before
// the launch) and the BabyBear twiddle table its contiguous passes stage.
struct WorkPhase {
  std::vector<WorkItem> items;
  std::vector<WorkUnit> units;
  const uint2* bb_tw = nullptr;
};

// Items that the persistent phases run: BabyBear or M31, 2^13..2^21 points,
// blow-up <= 16, TMA-aligned buffers, the default TMA plan, and no more tiles
// than the context's worklist_max_tiles (larger items fill the GPU alone).
bool worklist_eligible(const sfntt_ctx* ctx, const sfntt_lde_item& it);
// Appends the item's pass of `phase` (0: inverse layers [0, log n - 8),
// 1: expansion, 2: forward layers [0, log n - 8) of the extended network).
Status worklist_add(sfntt_ctx* ctx, WorkPhase& ph, int phase, const sfntt_lde_item& it, cudaStream_t s);
// One launch of `phase` over the device copy of ph (counter zeroed first).
Status worklist_launch(sfntt_ctx* ctx, int phase, const WorkPhase& ph, const WorkItem* items, const WorkUnit* units,
                       uint32_t* counter, cudaStream_t s);

}  // namespace sfntt
