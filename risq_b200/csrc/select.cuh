// Heat-bath excitation tables and the device selection step (select.cu, hci.cu).
#pragma once
#include <cstdint>
#include <vector>

#include "internal.cuh"

namespace risq {

// ExciteGenerator (src/excite/init.rs:33-58) flattened: list (p, q) of opposite-spin
// doubles is entries [opp_off[p*n+q], opp_off[p*n+q+1]), same-spin doubles (p < q)
// [same_off[p*n+q], ...), singles from p [sing_off[p], sing_off[p+1]); each list is in
// the reference's order (decreasing |H|, stable).
struct SelectTables {
    std::vector<int32_t> opp_off, same_off, sing_off;
    std::vector<uint8_t> r, s;
    std::vector<double> habs;
    double max_opp = 0.0, max_same = 0.0, max_sing = 0.0;
    uint64_t valence[2] = {0, 0};
    std::vector<int> valence_orbs, core_orbs;
};

struct SelectStats {
    uint64_t candidates = 0;  // excitations above eps whose target is not in the space
    uint64_t unique = 0;      // first occurrences among them
    uint64_t added = 0;       // determinants appended (with spin flips)
};

int build_select_tables(risqgpu* h, int ncore, int n_up, int n_dn, SelectTables& t);
int find_new_dets_impl(risqgpu* h, const double* coeffs, double eps, bool singles, const SelectTables& tab,
                       std::vector<uint64_t>& new_dets, std::vector<double>& new_diag, SelectStats* st);

}  // namespace risq
