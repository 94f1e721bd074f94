// ne2b_step_kind.h — the step kernels by kind (internal).  Each of the four
// kinds (int32 or f32 ring) x (with or without the AdEx path) is compiled in
// its own translation unit (ne2b_step_k*.cu) so the kernel instances build in
// parallel; ne2b_kernels.cu dispatches to them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_layout.h"

// Tile shapes compiled in: (threads per block, neurons per thread).
#define NE2B_SHAPES(X) \
    X(64, 1) X(64, 2) X(64, 4) X(128, 1) X(128, 2) X(128, 4) X(128, 8) X(256, 1) X(256, 2) X(256, 4) X(256, 8) \
    X(512, 1) X(512, 2) X(512, 4)
// Shapes with an instance of the warp-specialised single-net kernel
// (step_kernel_ws: the tile warps plus separate delivery warps).
#define NE2B_WS_SHAPES(X) \
    X(128, 1) X(128, 2) X(128, 4) X(128, 8) X(256, 1) X(256, 2) X(256, 4) X(256, 8) X(512, 1) X(512, 2) X(512, 4)

namespace ne2b {

bool pdl_enabled();  // programmatic dependent launch of the streaming kernels (ne2b_kernels.cu)

// 32-bit words of the delivery phase's shared lists (SmemLists).
template <int BLOCK, int NPT>
__host__ __device__ constexpr uint32_t smem_lists_words() {
    return 2 * BLOCK * NPT + 1 + 2 * (BLOCK / 32) + 2;
}

// Resident kernel shared memory: [delivery lists][flag u32], 16-byte aligned,
// then the owned state [v M f32][u M f32][s M f32][tk M u16][pidx M u16].
template <int BLOCK, int NPT>
__host__ __device__ constexpr uint32_t resident_head_bytes() {
    return (uint32_t)((smem_lists_words<BLOCK, NPT>() + 1) * 4 + 15) / 16 * 16;
}

// Streaming kernel instances: one net with any features, one net without the
// optional ones (external current, stimulus, records, windows, custom-tau
// synapses, f32 trace, watches), many nets (batches, the server), and many
// nets without records, custom-tau synapses, f32 trace or watches.
enum StepVariant : int { kStepSingle = 0, kStepMulti = 1, kStepPlain = 2, kStepMultiLean = 3 };
// Added to kStepSingle or kStepPlain: the warp-specialised instance
// (separate delivery warps; engines of one net, NE2B_WS_SHAPES only).
constexpr int kStepWS = 0x10;

template <bool INT, bool ADEX>
struct StepKind {
    static int occupancy(uint32_t block, uint32_t npt, int variant);
    static cudaError_t launch(uint32_t block, uint32_t npt, int variant, const EngineDev *eng, uint32_t k_step,
                              uint32_t grid, cudaStream_t st);
    static int resident_occupancy(uint32_t block, uint32_t npt, size_t smem);
    static cudaError_t launch_resident(uint32_t block, uint32_t npt, const EngineDev *eng, uint32_t k0,
                                       uint32_t nsteps, uint32_t grid, size_t smem, cudaStream_t st);
};
extern template struct StepKind<false, false>;
extern template struct StepKind<false, true>;
extern template struct StepKind<true, false>;
extern template struct StepKind<true, true>;

}  // namespace ne2b
