// Nuclear attraction V[mu nu C] with the fast kernels: point-charge ket
// (lane = charge), every fast pair class, FP64.  Variant 3 (no register cap)
// for the d-d and p-d pairs, whose 16-warp cap of variant 0 spills; variant 0
// elsewhere.
#include "k3c_fast.cuh"

namespace eip {

int launch_fast_point(int li, int lj, const BraTable& bra, const KetTable& ket, const BatchMap& map,
                      int total_items, double omega, double* out, int* counter, cudaStream_t s) {
    const double* t = boys_table_device();
    if (!t) return 2;
#define EIP_P(I, J) \
    return launch_one<I, J, 0, (I + J >= 3 ? 3 : 0), double, true>(t, bra, ket, map, total_items, omega, out, counter, s)
    switch (li * 10 + lj) {
        case 0: EIP_P(0, 0);
        case 1: EIP_P(0, 1);
        case 11: EIP_P(1, 1);
        case 2: EIP_P(0, 2);
        case 12: EIP_P(1, 2);
        case 22: EIP_P(2, 2);
        case 3: EIP_P(0, 3);
        case 4: EIP_P(0, 4);
    }
#undef EIP_P
    return 1;
}

}  // namespace eip
