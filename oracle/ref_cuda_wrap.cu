/*
 * ref_cuda_wrap.cu -- C entry points onto the reference's own CUDA kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
 * src/cuda/aco_cuda_kernels.cu from the reference sources (for sm_100a) into
 * oracle/_ref/librefcuda.so.  The GPU parity tests run these kernels and the
 * product's kernels on the same device buffers and compare bytes: the
 * reference's quantize/dequantize use device expf/logf
 * (aco_cuda_kernels.cu:25-45), which only the same device math reproduces.
 *
 * The launch_* wrappers (aco_cuda_kernels.cu:678-772) run on the default
 * stream; each entry point synchronizes and returns the CUDA error code.
 */
#include "aco_cuda_kernels.h"

#include <cuda_runtime.h>

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

REF_EXPORT int refcuda_init_tau(uint8_t *d_tau, int n, uint8_t q_tau0) {
  launch_init_tau(d_tau, n, q_tau0);
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int refcuda_evaporate(uint8_t *d_tau, int n, uint8_t delta,
                                 uint8_t q_min) {
  launch_evaporate_tau(d_tau, n, delta, q_min);
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int refcuda_build_candidates(const float *d_coords_xy,
                                        int *d_candidate_idx,
                                        float *d_eta_beta,
                                        const CudaParams *params) {
  launch_build_candidate_lists((const float2 *)d_coords_xy, d_candidate_idx,
                               d_eta_beta, *params);
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int refcuda_deposit_solution(uint8_t *d_tau, const int *d_routes,
                                        const int *d_route_lengths,
                                        float deposit_amount, int best_ant,
                                        const CudaParams *params) {
  launch_deposit_solution(d_tau, d_routes, d_route_lengths, deposit_amount,
                          best_ant, *params);
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int refcuda_deposit_flat(uint8_t *d_tau, const int *d_flat_routes,
                                    const int *d_flat_lengths,
                                    float deposit_amount,
                                    const CudaParams *params) {
  launch_deposit_flat_solution(d_tau, d_flat_routes, d_flat_lengths,
                               deposit_amount, *params);
  return (int)cudaDeviceSynchronize();
}

REF_EXPORT int refcuda_params_size(void) { return (int)sizeof(CudaParams); }
