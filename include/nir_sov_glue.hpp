// Shared state of the drop-in headers (nirnaya_b200/sov/*.hpp), C++ only.
//
// Solver::solve scales the presolved model with scale_model and hands the
// scaled model to PdhgSolver::solve (include/sov/solver.hpp:180-244).  The
// drop-in scale_model records its scales here.  The drop-in PdhgSolver undoes
// them before the engine runs: the engine equilibrates by itself, and
// rescaling ahead of it slows the restarted PDHG's duality gap.  The scales
// are powers of two, so undoing them is exact.  Any positive diagonal
// rescaling gives an equivalent LP, so the solution mapped back is a
// solution of the model PdhgSolver was given, whatever model that is.
#pragma once

#include <vector>

namespace nir {
namespace sov_glue {

struct LastScaling {
    bool active = false;
    std::vector<double> R;  // row scales of the last scale_model call on this thread
    std::vector<double> C;  // column scales
};

inline LastScaling& last_scaling() {
    thread_local LastScaling s;
    return s;
}

}  // namespace sov_glue
}  // namespace nir
