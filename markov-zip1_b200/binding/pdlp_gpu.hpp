// The GPU module of markov-cero's first-order LP path: solve_pdlp for
// Backend::gpu on the B200 engine (libmcpdlp.so, include/mc_pdlp.h).
//
// This is the "src/gpu" module a maintainer adds to the reference solver.  It
// takes the reference's own types -- model::Model
// (include/markov_cero/model/model.hpp:53-70), PdlpOptions and PdlpResult
// (include/markov_cero/lp/first_order/pdlp.hpp:18-63) -- and keeps the
// reference's error classes: malformed input throws std::invalid_argument,
// sizes beyond the engine's int32 indices throw std::length_error, anything
// else (no B200, CUDA failure) throws std::runtime_error.  These are the
// three classes the CLI maps to InvalidModel / ResourceLimit /
// NumericalFailure (apps/markov_cero_solve.cpp:418-434).  There is no CPU
// fallback: backend_actually_used is always "cuda".
#pragma once

#include "markov_cero/lp/first_order/pdlp.hpp"
#include "markov_cero/model/model.hpp"

namespace markov_cero::gpu {

// The GPU solve (the reference's solve_pdlp contract, pdlp.hpp:67).
[[nodiscard]] lp::first_order::PdlpResult solve_pdlp_gpu(const model::Model& model,
                                                         const lp::first_order::PdlpOptions& options);

// True when this solve goes to the GPU: options.backend == Backend::gpu, or
// the process-wide switch MARKOV_CERO_PDLP_BACKEND=gpu is set (it routes every
// solve_pdlp of the process to the GPU, so that existing tools and test
// programs run on the GPU without changes to their option code).
[[nodiscard]] bool gpu_requested(const lp::first_order::PdlpOptions& options);

}  // namespace markov_cero::gpu
