// solve_pdlp with the GPU backend dispatched to the B200 engine.
//
// The reference's entry (src/lp/first_order/pdlp.cpp:139) runs the CPU solver
// for every backend and labels a GPU request "cpu_fallback".  This file is
// the entry the integrated solver exports instead: a GPU request goes to
// markov_cero::gpu::solve_pdlp_gpu, everything else to the reference's CPU
// body, which the integration build compiles under the name
// solve_pdlp_cpu (pdlp.cpp built with -Dsolve_pdlp=solve_pdlp_cpu), so no
// reference source is edited.  In a maintainer's tree the same three lines
// sit at the top of solve_pdlp itself.
#include "markov_cero/lp/first_order/pdlp.hpp"
#include "pdlp_gpu.hpp"

namespace markov_cero::lp::first_order {

PdlpResult solve_pdlp_cpu(const model::Model& model, const PdlpOptions& options);

PdlpResult solve_pdlp(const model::Model& model, const PdlpOptions& options) {
    if (gpu::gpu_requested(options)) return gpu::solve_pdlp_gpu(model, options);
    return solve_pdlp_cpu(model, options);
}

}  // namespace markov_cero::lp::first_order
