// Prints the serving loop's launch form for argument tuples read from stdin:
// "split take busy sm_count conc4 conc2" -> serve_split, "blocks split take conc"
// -> serve_blocks. Used by tests/test_serve_policy_cpu.py (no GPU).
#include <cstdint>
#include <iostream>
#include <string>

#include "serve_policy.h"

int main() {
    std::string op;
    while (std::cin >> op) {
        if (op == "split") {
            uint64_t take, busy, sms, c4, c2;
            std::cin >> take >> busy >> sms >> c4 >> c2;
            std::cout << tp::serve_split(take, busy, sms, c4, c2) << "\n";
        } else if (op == "blocks") {
            int split;
            uint64_t take, conc;
            std::cin >> split >> take >> conc;
            std::cout << tp::serve_blocks(split, take, conc) << "\n";
        } else {
            return 2;
        }
    }
    return 0;
}
