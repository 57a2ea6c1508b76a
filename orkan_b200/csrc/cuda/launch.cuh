// launch.cuh - launch helpers shared by the translation units of the kernel layer:
// the SM count of the current device, grid sizing, the counted launch check, and the
// density-matrix phase-pass launcher used by gates and exp_diag.
#pragma once

#include "common.cuh"
#include "dm_phase.cuh"

namespace orkan {

// Multiprocessors of the current device (cached per device; 148 on B200).
int sm_count();

// Counts one kernel launch (orkan_cu_launch_count) and returns the launch status.
int finish_launch();

// Grid cap of the streaming kernels: one block per share of work, no persistent loop.  The
// blocks are scheduled by the hardware as SMs free up, which measured 15 % faster at 30
// qubits than grid-stride loops over 8 blocks per SM (the register use of those kernels
// leaves room for four 256-thread blocks per SM, so such a grid ran in two rounds).
constexpr unsigned kFullGrid = 0x7fffffffu;

// Blocks for total_units of work at work_per_block_units per block, at least 1, at most cap.
inline unsigned grid_for(idx_t work_per_block_units, idx_t total_units, unsigned cap) {
    idx_t g = (total_units + work_per_block_units - 1) / work_per_block_units;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

// Items (S x S sub-tiles) per block of the phase pass: 2, or 1 / 4 / 8 through the tuning
// knob ORKAN_PHASE_ITEMS, read once.
unsigned phase_items_per_block();

// Elementwise phase pass over a packed (layout 1) or tiled (layout 2) density matrix.
template <class Factor>
int launch_phase(int layout, unsigned log_tile, void* rho, unsigned n, const Factor& fac, cudaStream_t st) {
    const PhaseGeom g = phase_geometry(n, layout == 2 ? log_tile : 5u);
    const unsigned grid = grid_for(phase_items_per_block(), g.items, kFullGrid);
    DevMem mem{static_cast<double2*>(rho)};
    if (layout == 1) {
        k_dm_phase<PackedMap, Factor><<<grid, kPhaseThreads, 0, st>>>(mem, PackedMap{idx_t(1) << n}, g, fac);
    } else {
        k_dm_phase<TiledMap, Factor><<<grid, kPhaseThreads, 0, st>>>(mem, TiledMap{idx_t(1) << n, log_tile}, g, fac);
    }
    return finish_launch();
}

}  // namespace orkan
