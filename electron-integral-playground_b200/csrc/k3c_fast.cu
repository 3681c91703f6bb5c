// Dispatcher of the fast (mu nu|P) kernels; one translation unit per (l_i, l_j)
// (k3c_fast_IJ.cu) so the template instances compile in parallel.
#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

#define EIP_DECL(I, J) \
    int launch_fast3c_##I##J(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket, \
                             double omega, double* out, cudaStream_t s);
EIP_DECL(0, 0) EIP_DECL(0, 1) EIP_DECL(1, 1) EIP_DECL(0, 2) EIP_DECL(1, 2) EIP_DECL(2, 2)
#undef EIP_DECL

bool fast3c_supported(int li, int lj, int lk) {
    return li >= 0 && li <= lj && lj <= 2 && lk >= 0 && lk <= 4;
}

int launch_fast3c(int li, int lj, int lk, const BraTable& bra, const KetTable& ket, double omega, double* out,
                  cudaStream_t s) {
    const double* t = boys_table_device();
    switch (li * 10 + lj) {
        case 0: return launch_fast3c_00(lk, t, bra, ket, omega, out, s);
        case 1: return launch_fast3c_01(lk, t, bra, ket, omega, out, s);
        case 11: return launch_fast3c_11(lk, t, bra, ket, omega, out, s);
        case 2: return launch_fast3c_02(lk, t, bra, ket, omega, out, s);
        case 12: return launch_fast3c_12(lk, t, bra, ket, omega, out, s);
        case 22: return launch_fast3c_22(lk, t, bra, ket, omega, out, s);
    }
    return 1;
}

}  // namespace eip
