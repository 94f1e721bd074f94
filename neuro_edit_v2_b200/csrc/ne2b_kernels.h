// ne2b_kernels.h — host-side launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ne2b_layout.h"

namespace ne2b {

bool shape_supported(uint32_t block, uint32_t npt);
bool ws_shape_supported(uint32_t block, uint32_t npt);  // step_kernel_ws compiled for this shape
void set_pdl(bool on);  // programmatic dependent launch of the streaming kernels (default on)
void shape_list(uint32_t *blocks, uint32_t *npts, uint32_t *count);
// `adex`: an AdEx row is present in some net (else the Izhikevich-only
// instance of the step kernels runs).  `variant` (StepVariant): kStepMulti
// when the engine holds many nets (a batch or the server), whose streaming
// kernel stages several tiles' records and net descriptors ahead; kStepPlain
// for one net without the optional features; else kStepSingle.
int step_occupancy(bool int_ring, bool adex, int variant, uint32_t block, uint32_t npt);
// k_step > 0 launches are programmatic (they follow step k_step - 1 of the
// same launch group); k_step = 0 follows advance_kernel or host copies and
// waits for them in full.
cudaError_t launch_step(bool int_ring, bool adex, int variant, uint32_t block, uint32_t npt, const EngineDev *eng,
                        uint32_t k_step, uint32_t grid, cudaStream_t st);
uint32_t resident_head(uint32_t block, uint32_t npt);
int resident_occupancy(bool int_ring, bool adex, uint32_t block, uint32_t npt, size_t smem);
cudaError_t launch_resident(bool int_ring, bool adex, uint32_t block, uint32_t npt, const EngineDev *eng,
                            uint32_t k0, uint32_t nsteps, uint32_t grid, size_t smem, cudaStream_t st);
cudaError_t launch_advance(NetDev *nets, uint32_t n_nets, uint32_t steps, cudaStream_t st);
// Bounded grid barrier self-test: `blocks` cooperative blocks of which
// `absent` never arrives; the others stop after `limit_ns` and set *err.
cudaError_t launch_barrier_selftest(unsigned int *counter, unsigned int *err, uint32_t blocks, uint32_t absent,
                                    unsigned long long limit_ns, cudaStream_t st);
cudaError_t launch_reset_neurons(const NetDev &nd, cudaStream_t st);
cudaError_t launch_trace(const uint16_t *tk, const float *tab, uint32_t n, float *out, cudaStream_t st);
cudaError_t launch_window_count(const uint32_t *rec_bits, uint32_t rec_rows, uint32_t n_pad, uint32_t n,
                                unsigned long long t, uint32_t rows, uint32_t *out, cudaStream_t st);
cudaError_t launch_pn_total(const unsigned long long *pn, uint32_t n, uint32_t *out, cudaStream_t st);

}  // namespace ne2b
