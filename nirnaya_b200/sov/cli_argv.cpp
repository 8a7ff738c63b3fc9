// The CLI's program entry for the drop-in build of `sovsolve`.
//
// The reference's README advertises `--method=auto|simplex|ipm|pdhg`
// (its README.md:27), but its argument loop only takes the two-token form
// `--method pdhg` (src/driver/cli_main.cpp:51-52) and silently skips any
// other dash argument (:77), so `--method=pdhg` ran the dual simplex.
// This entry splits every `--<option>=<value>` of an option that takes a
// value into `--<option> <value>` and hands the result to the reference's
// own main, which the Makefile compiles under the name below.  Nothing
// else changes: unknown options, the two-token forms and `--set name=value`
// reach the reference's loop exactly as given.
#include <cstring>
#include <string>
#include <vector>

int sov_reference_cli_main(int argc, char** argv);

namespace {

// The options of src/driver/cli_main.cpp:41-76 that read the next token.
const char* const kValued[] = {"--sol",     "--stats-json", "--time-limit", "--threads",     "--method",
                               "--presolve", "--mip-gap",   "--mip-abs-gap", "--node-limit", "--seed",
                               "--log",      "--tolerance-preset", "--set"};

bool takes_value(const std::string& name) {
    for (const char* v : kValued)
        if (name == v) return true;
    return false;
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> args;
    args.reserve(size_t(argc) + 4);
    for (int i = 0; i < argc; ++i) {
        const std::string a = argv[i];
        const size_t eq = a.find('=');
        if (i > 0 && a.size() > 2 && a[0] == '-' && a[1] == '-' && eq != std::string::npos &&
            takes_value(a.substr(0, eq))) {
            args.push_back(a.substr(0, eq));
            args.push_back(a.substr(eq + 1));
        } else {
            args.push_back(a);
        }
    }
    std::vector<char*> av;
    av.reserve(args.size() + 1);
    for (auto& s : args) av.push_back(&s[0]);
    av.push_back(nullptr);
    return sov_reference_cli_main(int(args.size()), av.data());
}
