// ref_sol_tool.cpp -- the reference's SolIo::read_sol (src/io/sol_io.hpp:
// 134-170) as a program, compiled from the reference's sources in place
// (oracle/Makefile, output oracle/_ref/ref_sol_tool).
//
// TEST INFRASTRUCTURE ONLY.  read_sol extracts values with istream >>
// double, which fails when this code runs as a library inside the Python
// process of the tests (its statically linked C++ runtime), so the tests run
// it as its own process:
//   ref_sol_tool <model.mps> <solution.sol>
// prints "status <n>" and "objective <hex>", then one "<j> <hex>" line per
// column, or "exception <what>" when an exception escapes read_sol, or
// "cannot-open" when read_sol returns false.
#include "include/sov/solver.hpp"

#include <cstdio>

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    sov::Model m;
    std::string err;
    if (sov::MpsReader::read(argv[1], m, err) != sov::Status::Optimal) {
        std::printf("model-error %s\n", err.c_str());
        return 3;
    }
    sov::Status st;
    double obj = 0.0;
    std::vector<double> x;
    try {
        if (!sov::SolIo::read_sol(argv[2], m, st, obj, x)) {
            std::printf("cannot-open\n");
            return 0;
        }
    } catch (const std::exception& e) {
        std::printf("exception %s\n", e.what());
        return 0;
    }
    std::printf("status %d\nobjective %a\n", static_cast<int>(st), obj);
    for (size_t j = 0; j < x.size(); ++j) std::printf("%zu %a\n", j, x[j]);
    return 0;
}
