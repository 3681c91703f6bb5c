// One compiled instance of the fast (mu nu|P) kernels: pair class
// (l_i, l_j) = (EIP_LI, EIP_LJ), tuning variant EIP_V, arithmetic type
// double (EIP_FP32 = 0) or float (EIP_FP32 = 1, the mixed-precision path),
// every l_k = 0..4.  The Makefile compiles this file once per instance with
// those four -D flags, so the instances compile in parallel; the result
// defines launch_fast3c_<li><lj>_v<V> or launch_fast3c_<li><lj>_f32_v<V>
// (declared and dispatched in k3c_fast.cu), and the variant-0 FP64 instance
// also the pair class's E-table launcher launch_e_table_<li><lj>.
#include <type_traits>

#include "k3c_fast.cuh"

#if !defined(EIP_LI) || !defined(EIP_LJ) || !defined(EIP_V) || !defined(EIP_FP32)
#error "k3c_fast_inst.cu needs -DEIP_LI, -DEIP_LJ, -DEIP_V and -DEIP_FP32"
#endif

#define EIP_CAT_(a, b) a##b
#define EIP_CAT(a, b) EIP_CAT_(a, b)
#define EIP_PAIR EIP_CAT(EIP_LI, EIP_LJ)
#if EIP_FP32
#define EIP_LAUNCH EIP_CAT(EIP_CAT(EIP_CAT(launch_fast3c_, EIP_PAIR), _f32_v), EIP_V)
#else
#define EIP_LAUNCH EIP_CAT(EIP_CAT(EIP_CAT(launch_fast3c_, EIP_PAIR), _v), EIP_V)
#endif

namespace eip {

int EIP_LAUNCH(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket, const BatchMap& map,
               int total_items, double omega, double* out, int* counter, cudaStream_t s) {
    using T = std::conditional_t<EIP_FP32 != 0, float, double>;
    switch (lk) {
        case 0: return launch_one<EIP_LI, EIP_LJ, 0, EIP_V, T>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 1: return launch_one<EIP_LI, EIP_LJ, 1, EIP_V, T>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 2: return launch_one<EIP_LI, EIP_LJ, 2, EIP_V, T>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 3: return launch_one<EIP_LI, EIP_LJ, 3, EIP_V, T>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
        case 4: return launch_one<EIP_LI, EIP_LJ, 4, EIP_V, T>(boys_table, bra, ket, map, total_items, omega, out, counter, s);
    }
    return 1;
}

#if EIP_V == 0 && !EIP_FP32
int EIP_CAT(launch_e_table_, EIP_PAIR)(const BraTable& bra, double* prim_E, cudaStream_t s) {
    return launch_e_table<EIP_LI, EIP_LJ>(bra, prim_E, s);
}
#endif

}  // namespace eip
