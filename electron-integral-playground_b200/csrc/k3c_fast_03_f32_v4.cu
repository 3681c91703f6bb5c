// Mixed-precision (FP32 R/ket/bra) (mu nu|P) instances for (l_i, l_j) = (0, 3),
// l_k = 0..4 (tuning variant 4).
#include "k3c_fast.cuh"

namespace eip {

int launch_fast3c_03_f32_v4(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket,
                          const BatchMap& map, int total_items, double omega, double* out, int* counter,
                          cudaStream_t s) {
    switch (lk) {
        case 0: return launch_one<0, 3, 0, 4, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 1: return launch_one<0, 3, 1, 4, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 2: return launch_one<0, 3, 2, 4, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 3: return launch_one<0, 3, 3, 4, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 4: return launch_one<0, 3, 4, 4, float>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
    }
    return 1;
}

}  // namespace eip
