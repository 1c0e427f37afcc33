// The GPU module of markov-cero's canonical-model presolve: presolve() and
// postsolve() (include/markov_cero/presolve/presolve.hpp:39-45) on the B200
// engine (mc_presolve_run / mc_postsolve, include/mc_pdlp.h).
//
// Same types, results and errors as the reference's functions: the input is
// checked by the reference's own SparseCanonicalModel::validate (so its size
// cap and exceptions are kept), the reduced model by validate() as
// presolve.cpp:211-213 does, and postsolve throws std::overflow_error on a
// non-finite dual or objective as presolve.cpp:297-298 and :307 do.  Anything
// else (no B200, CUDA failure) throws std::runtime_error; there is no CPU
// fallback.  A maintainer routes callers here, or compiles them with the
// function-like macros presolve(...) -> presolve_gpu(...) and postsolve(...)
// -> postsolve_gpu(...), which leave the namespace markov_cero::presolve
// untouched (a function-like macro expands only before "(").
#pragma once

#include "markov_cero/lp/reference/revised_simplex.hpp"
#include "markov_cero/presolve/presolve.hpp"
#include "markov_cero/transform/sparse_canonical_model.hpp"

namespace markov_cero::presolve {

[[nodiscard]] PresolveResult presolve_gpu(const transform::SparseCanonicalModel& input,
                                          const PresolveOptions& options = {});

[[nodiscard]] lp::reference::Result postsolve_gpu(const PresolveStack& stack,
                                                  const lp::reference::Result& reduced_solution,
                                                  const transform::SparseCanonicalModel& original_model,
                                                  double tolerance = 1e-8);

}  // namespace markov_cero::presolve
