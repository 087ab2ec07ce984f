// Writes ke_pattern.inc (to stdout): the coefficient pattern of the built-in hex8 Ke used by the FP64
// streaming K(E)u.
//
// The 576 entries of hex8_stiffness(0.3, 1.0) take only KE_ND distinct magnitudes (bit for bit).  The
// kernel keeps those magnitudes in registers and reads each coefficient as +-D[ke_idx(i)], so every DFMA
// has register operands only; the sign is the operand's negation, which is exact.  ke_row_order lists,
// for each column j, the 24 rows sorted by magnitude index, so that consecutive DFMAs of one column share
// their coefficient register (the rows are independent chains, so their order changes no result).
// At run time the library checks a context's Ke against this pattern and uses the generic kernel when it
// does not match (e.g. after t3d_set_ke).
//
// Build and run:  g++ -std=c++17 -O2 gen_ke_pattern.cpp -o gen && ./gen > ke_pattern.inc
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "hex8.hpp"

static void table(const char* name, const char* type, const std::vector<int>& v) {
    std::printf("__host__ __device__ constexpr int %s(int i) {\n    constexpr %s t[%zu] = {", name, type, v.size());
    for (size_t i = 0; i < v.size(); ++i) std::printf("%s%s%d", i ? "," : "", i % 32 == 0 ? "\n        " : "", v[i]);
    std::printf("};\n    return t[i];\n}\n");
}

int main() {
    double Ke[576];
    t3d::hex8_stiffness(0.3, 1.0, Ke);
    std::vector<double> mags;
    std::vector<int> idx(576), neg(576), first;
    for (int i = 0; i < 576; ++i) {
        const double m = std::fabs(Ke[i]);
        auto it = std::find(mags.begin(), mags.end(), m);
        if (it == mags.end()) {
            mags.push_back(m);
            first.push_back(i);
            it = mags.end() - 1;
        }
        idx[i] = (int)(it - mags.begin());
        neg[i] = Ke[i] < 0.0 ? 1 : 0;
    }
    std::vector<int> order;
    for (int j = 0; j < 24; ++j) {
        std::vector<int> rows(24);
        for (int q = 0; q < 24; ++q) rows[q] = q;
        std::stable_sort(rows.begin(), rows.end(), [&](int a, int b) {
            const int ia = idx[a * 24 + j], ib = idx[b * 24 + j];
            return ia != ib ? ia < ib : neg[a * 24 + j] < neg[b * 24 + j];
        });
        order.insert(order.end(), rows.begin(), rows.end());
    }
    std::printf("// Generated by gen_ke_pattern.cpp from hex8_stiffness(0.3, 1.0); do not edit.\n");
    std::printf("// Ke[i] == (ke_neg(i) ? -1 : 1) * |Ke[ke_first(ke_idx(i))]| for i = 24 * row + column.\n");
    std::printf("#pragma once\n\nconstexpr int KE_ND = %zu;\n", mags.size());
    table("ke_idx", "unsigned char", idx);
    table("ke_neg", "unsigned char", neg);
    table("ke_first", "short", first);
    table("ke_row_order", "unsigned char", order);
    return 0;
}
