// Fast (mu nu|P) instances for (l_i, l_j) = (1, 1), l_k = 0..4.
#include "k3c_fast.cuh"

namespace eip {

int launch_fast3c_11(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket, double omega,
                        double* out, cudaStream_t s) {
    switch (lk) {
        case 0: return launch_one<1, 1, 0>(boys_table, bra, ket, omega, out, s);
        case 1: return launch_one<1, 1, 1>(boys_table, bra, ket, omega, out, s);
        case 2: return launch_one<1, 1, 2>(boys_table, bra, ket, omega, out, s);
        case 3: return launch_one<1, 1, 3>(boys_table, bra, ket, omega, out, s);
        case 4: return launch_one<1, 1, 4>(boys_table, bra, ket, omega, out, s);
    }
    return 1;
}

}  // namespace eip
