// The GPU module of markov-cero's canonical-model scaling: equilibrate()
// (include/markov_cero/scale/ruiz_scaling.hpp:28-29,
// src/scale/ruiz_scaling.cpp:20-125) on the B200 engine
// (mc_ruiz_equilibrate_canonical, include/mc_pdlp.h).  Same arguments and
// result: the model's values, rhs and objective are scaled in place and the
// scales come back in RuizScalers; the device result is bit-identical.  The
// engine also checks the CSC (sorted rows, no explicit zeros, finite values)
// and throws std::invalid_argument where it is malformed; no B200 or a CUDA
// failure throws std::runtime_error (there is no CPU fallback).  Callers can
// be compiled with the function-like macro equilibrate(...) ->
// equilibrate_gpu(...), which leaves equilibrate_model untouched.
#pragma once

#include "markov_cero/scale/ruiz_scaling.hpp"
#include "markov_cero/transform/sparse_canonical_model.hpp"

namespace markov_cero::scale {

[[nodiscard]] RuizScalers equilibrate_gpu(transform::SparseCanonicalModel& model, const RuizOptions& options = {});

}  // namespace markov_cero::scale
