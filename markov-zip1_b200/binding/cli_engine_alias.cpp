// The `--engine pdlp-gpu` option of markov-cero-solve.
//
// The reference CLI already routes `--engine pdlp --backend gpu` to
// solve_pdlp with Backend::gpu (apps/markov_cero_solve.cpp:136-140,
// apps/cli_options.hpp:218-229).  `pdlp-gpu` names that pair as one engine:
// this entry rewrites it and hands the arguments to the CLI's own main, which
// the integration build compiles as markov_cero_solve_main
// (-Dmain=markov_cero_solve_main).  A maintainer's tree instead adds
// "pdlp-gpu" to the engine whitelist (apps/cli_options.hpp:85-89) and sets
// the backend where the engine is resolved.
#include <cstring>
#include <string>
#include <vector>

int markov_cero_solve_main(int argc, char** argv);

int main(int argc, char** argv) {
    std::vector<std::string> args(argv, argv + argc);
    std::vector<std::string> out;
    out.reserve(args.size() + 2);
    bool gpu = false;
    for (std::size_t i = 0; i < args.size(); ++i) {
        if (args[i] == "--engine" && i + 1 < args.size() && args[i + 1] == "pdlp-gpu") {
            out.push_back("--engine");
            out.push_back("pdlp");
            gpu = true;
            ++i;
            continue;
        }
        out.push_back(args[i]);
    }
    if (gpu) {
        out.push_back("--backend");
        out.push_back("gpu");
    }
    std::vector<char*> ptrs;
    for (auto& s : out) ptrs.push_back(s.data());
    ptrs.push_back(nullptr);
    return markov_cero_solve_main(static_cast<int>(out.size()), ptrs.data());
}
