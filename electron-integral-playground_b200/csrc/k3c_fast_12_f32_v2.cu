// Mixed-precision (FP32 R/ket/bra) (mu nu|P) instances for (l_i, l_j) = (1, 2),
// l_k = 0..4 (tuning variant 2).
#include "k3c_fast.cuh"

namespace eip {

int launch_fast3c_12_f32_v2(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket,
                          const BatchMap& map, int total_items, double omega, double* out, int* counter,
                          cudaStream_t s) {
    switch (lk) {
        case 0: return launch_one<1, 2, 0, 2, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 1: return launch_one<1, 2, 1, 2, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 2: return launch_one<1, 2, 2, 2, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 3: return launch_one<1, 2, 3, 2, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 4: return launch_one<1, 2, 4, 2, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
    }
    return 1;
}

}  // namespace eip
