// kernels.h -- host-callable launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "kernels_common.cuh"

namespace rsr {

constexpr int kPlainThreads = 128;  // 4 warps per block, one work item per warp
constexpr int kRegThreads = 256;  // 8 warps share one work item
constexpr int kGradThreads = 32;  // one warp per block, one item per warp
// Points per partial sum: a program's MSE (and gradient) is the sum, in
// order, of its per-part sums, each part 4096 consecutive points of its
// dataset.  A work item covers one part (the register adjoint: up to
// kAdjMaxParts), so results do not depend on how a batch is cut into items.
constexpr uint32_t kPartPoints = 4096;
constexpr uint32_t kAdjMaxParts = 5;

cudaError_t launch_plain(const LaunchArgs &a, int P, uint32_t warps_per_block, size_t smem, cudaStream_t st);
size_t plain_smem_per_warp(uint32_t code_words, uint32_t const_floats, uint32_t slots, int P);
// Loads the slot-file kernel's variants and the MSE epilogue ahead of their
// first real launch (lazy module loading), with empty launches on st.
cudaError_t preload_plain_mse(cudaStream_t st);
// Every instance of the register, register-adjoint and slot-file adjoint
// kernels, loaded by empty launches (zero: a device word holding 0, the
// run_if that makes them return at once).  Module loading is lazy,
// and a kernel's first launch otherwise also resizes the context's local
// memory for its spills, which waits for all work on the device.
cudaError_t preload_reg(const uint32_t *zero, cudaStream_t st);
cudaError_t preload_adj(const uint32_t *zero, cudaStream_t st);
cudaError_t preload_grad(const uint32_t *zero, cudaStream_t st);
cudaError_t launch_aosoa_to_soa(const float *ff, const float *tb, float *x, float *y, uint32_t nf, uint64_t nbatch,
                                uint64_t stride, int num_sms, cudaStream_t st);
cudaError_t measure_fp32_peak(int num_sms, cudaStream_t st, double *lane_ops_per_s);
cudaError_t launch_finalize_sums(const ProgDesc *progs, const double *partials, uint32_t n, uint32_t stride,
                                 double *out, cudaStream_t st);
cudaError_t launch_finalize_mse(const ProgDesc *progs, const DatasetDesc *ds, const double *partials, uint32_t n,
                                float *out, cudaStream_t st);

// register-stack kernel (kernels_reg.cu)
// omit: handler sets the launch's programs do not need (bit 0: unary Float
// ops; bit 1: mat-vec with a feature, constant or spilled matrix), within
// reg_omittable(profile)
cudaError_t launch_reg(const LaunchArgs &a, int profile, int P, unsigned omit, uint32_t grid, cudaStream_t st);
unsigned reg_omittable(int profile);
void reg_layout(uint32_t code_words, uint32_t const_floats, const uint32_t *stack_depth, int P, int G,
                uint32_t *stack_off, uint32_t *acc_off, uint32_t *region_floats, uint32_t *block_hdr_floats);
int reg_max_p(int profile);
// Dynamic shared memory of one register-kernel block (bytes).
size_t reg_smem_bytes(uint32_t code_words, uint32_t const_floats, const uint32_t *stack_depth, int P, int G);
constexpr size_t kRegSmemBudget = 200 * 1024;  // at least one block per SM, below the 227 KB cap
int reg_max_blocks_per_sm(int profile, int P, unsigned omit, size_t smem);

// register adjoint (kernels_adj.cu): profiles F, F+V3, F+V2+M2, F+V3+M3;
// P (points per lane) 2, 4, or 8 up to adj_max_p(profile)
bool adj_supported(int profile);
int adj_max_p(int profile);
// floats of a warp's shared-memory region for a program (stacks, shared by
// the adjoint stacks | gradient sums | Kahan state), and its stack depths
// packed for ProgDesc
uint32_t adj_warp_floats(const uint32_t *stack_depth, int P, uint32_t n_params);
uint32_t adj_pack_depth(const uint32_t *stack_depth);
// shared-memory layout of a block of nw warps whose items cover at most
// `parts` parts; the tensor-memory columns of each warp's tape (512 / (nw /
// 4)) go to a->tmem_cols
void adj_layout(uint32_t code_words, uint32_t const_floats, uint32_t warp_floats, int nw, uint32_t parts,
                LaunchArgs *a);
size_t adj_smem_bytes(uint32_t code_words, uint32_t const_floats, uint32_t warp_floats, int nw, uint32_t parts);
// warps of a block of instance (profile, P), one block per SM (a multiple of 4)
int adj_block_warps(int profile, int P);
// Handler sets an instance may leave out (bit 0: unary Float ops; bit 1,
// F+V3: mat-vec with a leaf or spilled matrix), as for the register kernel.
unsigned adj_omittable(int profile);
cudaError_t launch_adj(const LaunchArgs &a, int profile, int P, unsigned omit, uint32_t grid, size_t smem,
                       cudaStream_t st);

// adjoint kernel (kernels_grad.cu)
cudaError_t launch_grad(const LaunchArgs &a, int profile, bool no_unary, uint32_t warps_per_block, size_t smem,
                        cudaStream_t st);
bool grad_has_no_unary(int profile);
size_t grad_smem_per_warp(uint32_t code_words, uint32_t const_floats, uint32_t val_slots, uint32_t adj_slots,
                          int P);
cudaError_t launch_finalize_grad(const ProgDesc *progs, const DatasetDesc *ds, const double *partials, uint32_t n,
                                 float *mse_out, float *grad_out, cudaStream_t st);

}  // namespace rsr
