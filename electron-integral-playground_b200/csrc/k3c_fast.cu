// Dispatcher of the fast (mu nu|P) kernels; one translation unit per (l_i, l_j)
// (k3c_fast_IJ.cu) so the template instances compile in parallel.
#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

#define EIP_DECL(I, J)                                                                                       \
    int launch_fast3c_##I##J(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket,     \
                             const BatchMap& map, int total_items, double omega, double* out, int* counter, \
                             cudaStream_t s);                                                                \
    int launch_e_table_##I##J(const BraTable& bra, double* prim_E, cudaStream_t s);
EIP_DECL(0, 0) EIP_DECL(0, 1) EIP_DECL(1, 1) EIP_DECL(0, 2) EIP_DECL(1, 2) EIP_DECL(2, 2)
#undef EIP_DECL

bool fast3c_supported(int li, int lj, int lk) {
    return li >= 0 && li <= lj && lj <= 2 && lk >= 0 && lk <= 4;
}

size_t e_table_doubles(int li, int lj) {
    size_t n = 0;
    for (int i = 0; i <= li; i++)
        for (int j = 0; j <= lj; j++) n += i + j + 1;
    return 3 * n;
}

int launch_fast3c(int li, int lj, int lk, const BraTable& bra, const KetTable& ket, const BatchMap& map,
                  int total_items, double omega, double* out, int* counter, cudaStream_t s) {
    const double* t = boys_table_device();
#define EIP_GO(I, J) return launch_fast3c_##I##J(lk, t, bra, ket, map, total_items, omega, out, counter, s)
    switch (li * 10 + lj) {
        case 0: EIP_GO(0, 0);
        case 1: EIP_GO(0, 1);
        case 11: EIP_GO(1, 1);
        case 2: EIP_GO(0, 2);
        case 12: EIP_GO(1, 2);
        case 22: EIP_GO(2, 2);
    }
#undef EIP_GO
    return 1;
}

int launch_e_table(int li, int lj, const BraTable& bra, double* prim_E, cudaStream_t s) {
    switch (li * 10 + lj) {
        case 0: return launch_e_table_00(bra, prim_E, s);
        case 1: return launch_e_table_01(bra, prim_E, s);
        case 11: return launch_e_table_11(bra, prim_E, s);
        case 2: return launch_e_table_02(bra, prim_E, s);
        case 12: return launch_e_table_12(bra, prim_E, s);
        case 22: return launch_e_table_22(bra, prim_E, s);
    }
    return 1;
}

}  // namespace eip
