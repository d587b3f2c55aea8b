// Internal interface of the batched (persistent, work-queue) aggregation.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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

struct BatchParams {
    const BatchInstanceDev* inst;
    const BatchItem* items;
    uint32_t num_items;
    uint32_t* cursor;             // work-queue head, zeroed before every launch
    uint32_t* status;
};

uint32_t batch_smem_bytes();
cudaError_t batch_prepare_launch();
cudaError_t launch_batch(const BatchParams& prm, uint32_t grid, cudaStream_t stream);
cudaError_t launch_batch_zero_outputs(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                      uint64_t total_groups, cudaStream_t stream);
cudaError_t launch_batch_finalize(const BatchInstanceDev* inst, const uint64_t* group_base, uint32_t ninst,
                                  uint64_t total_groups, cudaStream_t stream);

}  // namespace q1
