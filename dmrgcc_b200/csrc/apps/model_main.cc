// The reference's model executables, run on the GPU:
//   real_spinless_bose_square_model <input file>   (model/real_spinless_bose_square_model.cc)
//   complex_spinless_bose_square_model <input file> (model/complex_spinless_bose_square_model.cc)
//   complex_spinful_bose_square_model <input file> (model/complex_spinful_bose_square_model.cc)
//   real_spinful_bose_square_model <input file>    (the spinful model on real tensors; flux 0)
// Same argument, same input file, the same printed lines (the Got/Def echo of
// the keys aside): the sweep table, one energy per half-sweep, the total time.
// The optional keys precision, mode, seed, lanczos_tol and lanczos_graph of the
// input group choose the library's run options (dmrg_run_options_from_input);
// without them the run is the reference's.  Like the reference, a wrong
// argument count prints the usage and returns 0; an error that the reference
// would report by exit(-1) prints the library's message and returns 1.
#include <cstdio>

#include "dmrg_b200.hpp"

#ifndef DMRG_MODEL
#error "DMRG_MODEL names the model (real_spinless_bose_square, ...)"
#endif

int main(int argc, char* argv[]) {
    if (argc != 2) {
        std::printf("Usage: %s inputfile", argv[0]);
        return 0;
    }
    try {
        dmrg_run_options_t opt;
        dmrgcc_b200::check(dmrg_run_options_from_input(argv[1], &opt), "dmrg_run_options_from_input");
        dmrgcc_b200::Context ctx(0);
        dmrgcc_b200::RealTensorRundmrg run(ctx, argv[1], DMRG_MODEL, opt);
        run.Run();
    } catch (const dmrgcc_b200::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        std::fflush(stdout);
        return 1;
    }
    return 0;
}
