/*
 * mc_pdlp_testing.h -- test hooks of the PDLP engine (no counterpart in the
 * reference; not part of the solver API).
 *
 * They let the host-side failure paths be exercised without faulting a GPU.
 */
#ifndef MC_PDLP_TESTING_H
#define MC_PDLP_TESTING_H

#ifdef __cplusplus
extern "C" {
#endif

/* The next `count` device-arena allocations of any context fail as if
 * cudaMalloc had returned cudaErrorMemoryAllocation: the solve returns
 * MC_ERR_OUT_OF_MEMORY and no device memory is touched.  0 disarms. */
int mc_test_inject_alloc_failures(int count);

#ifdef __cplusplus
}
#endif

#endif
