// Test harness for the host-only row-block layout (nirnaya_b200/csrc/row_blocks.hpp).
// stdin:  cap count nrows  rp[0..nrows]  off[0..count]  [mode]
//   mode 0: build the batch layout and print it
//   mode 1: as 0, then corrupt descriptor k (next integer) and re-check
// stdout: "blocks b0.x b0.y ...", "owner ...", "lo ...", or "error <message>"
#include <cstdio>
#include <iostream>

#include "row_blocks.hpp"

int main() {
    int cap = 0, count = 0, nrows = 0;
    std::cin >> cap >> count >> nrows;
    std::vector<int> rp(nrows + 1), off(count + 1);
    for (auto& v : rp) std::cin >> v;
    for (auto& v : off) std::cin >> v;
    int mode = 0, k = 0;
    std::cin >> mode;
    if (mode == 1) std::cin >> k;
    try {
        std::vector<int> owner, lo;
        std::vector<int2> b = nir::build_batch_row_blocks(rp, off, cap, &owner, &lo);
        if (mode == 1) {
            b[k].y -= 1;
            nir::check_row_blocks(b, rp, cap);
        }
        std::printf("blocks");
        for (auto& d : b) std::printf(" %d %d", d.x, d.y);
        std::printf("\nowner");
        for (int o : owner) std::printf(" %d", o);
        std::printf("\nlo");
        for (int o : lo) std::printf(" %d", o);
        std::printf("\n");
    } catch (const std::exception& e) {
        std::printf("error %s\n", e.what());
    }
    return 0;
}
