// Internal interface of the batched (persistent, work-queue) aggregation.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace q1 {

constexpr uint32_t kBatchTileRows = 2048;

// Placement of one instance inside the batch kernel.
enum BatchMode : uint32_t {
    kModeRegisters = 0,   // num_groups <= 4: per-thread byte planes
    kModeShared = 1,      // shared-memory table: (group, discount) cells for <= 256 groups, else
                          // slots for keys < 2048 with the rest spilled to scratch
    kModeGlobal = 2,      // reductions straight into scratch
};

struct BatchInstanceDev {
    const uint8_t* col[6];        // ship, qty, disc, tax, price, key (16-byte aligned, device)
    uint64_t rows;
    int32_t cutoff;               // cutoff_day - 727563, clamped to [-1, 32767]
    uint32_t num_groups;
    uint32_t mode;                // BatchMode
    uint32_t pad;
    unsigned long long* acc;      // scratch: num_groups x 8 u64
    unsigned long long* out;      // caller's int128 table [num_groups][6][lo, hi]
};

struct BatchItem {
    uint32_t instance;
    uint32_t first_tile;
    uint32_t num_tiles;
    uint32_t pad;
};

// Engine that aggregates an instance inside the batch kernel (q1_keyagg.cuh).
enum BatchEngine : uint32_t {
    kEngRegisters = 0,   // PlaneRegs<4>
    kEngCube3 = 1,       // (group, discount, tax) cells, <= 64 groups
    kEngCube = 2,        // (group, discount) cells, <= 256 groups
    kEngSlots = 3,       // slots for keys < 2048, larger keys spilled
    kEngGlobal = 4,      // straight into scratch
    kEngines = 5,
};
uint32_t batch_engine(uint32_t mode, uint32_t num_groups);

// One execution runs two persistent kernels side by side: the register-planes kernel (queue 0)
// and the table kernel (queues 1..4, then it helps with queue 0 through the cells engine).
struct BatchParams {
    const BatchInstanceDev* inst;
    const BatchItem* items;             // grouped by engine: [item_begin[e], item_begin[e + 1])
    uint32_t item_begin[kEngines + 1];
    uint32_t role_end[kEngines];        // table kernel: CTAs [role_end[e-1], role_end[e]) start
                                        // with queue e (e = 1..4; role_end[0] = 0)
    uint32_t grid_regs, grid_tables;    // CTAs of the two kernels (a zero grid skips a kernel)
    uint32_t* cursor;                   // kEngines claim counters, zeroed before every launch
    uint32_t* status;
};

// Cuts every instance (host descriptors) into items of at most `chunk` tiles, groups them by
// engine (largest first inside an engine), splits the `grid` CTAs between the two kernels and
// the table kernel's among queues 1..4, in proportion to estimated cost.
void batch_plan(const BatchInstanceDev* inst, uint32_t n, uint32_t chunk, uint32_t grid, std::vector<BatchItem>& items,
                BatchParams& prm);

uint32_t batch_smem_bytes();
cudaError_t batch_prepare_launch();
// Launches the kernels of prm.grid_regs / prm.grid_tables; when both run, the register-planes
// kernel goes to `aux`, forked from and joined back into `stream` with the two events.
cudaError_t launch_batch(const BatchParams& prm, uint32_t grid_regs, uint32_t grid_tables, cudaStream_t stream,
                         cudaStream_t aux, cudaEvent_t fork, cudaEvent_t join);
cudaError_t launch_batch_zero_outputs(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                      uint64_t total_groups, cudaStream_t stream);
cudaError_t launch_batch_finalize(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                  uint64_t total_groups, cudaStream_t stream);

}  // namespace q1
