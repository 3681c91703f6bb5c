// Dispatcher of the fast (mu nu|P) kernels: one compiled instance per (l_i, l_j)
// pair class, tuning variant and type (k3c_fast_inst.cu, built once per
// instance by the Makefile) so the instances compile in parallel; the variant
// of each class comes from the tuning table (eip_tune_set).
#include "eip_common.cuh"
#include "eip_internal.h"

namespace eip {

#define EIP_DECL_V(I, J, V)                                                                                   \
    int launch_fast3c_##I##J##_v##V(int lk, const double* boys_table, const BraTable& bra, const KetTable& ket, \
                                    const BatchMap& map, int total_items, double omega, double* out,         \
                                    int* counter, cudaStream_t s);
#define EIP_DECL_F(I, J, V)                                                                                     \
    int launch_fast3c_##I##J##_f32_v##V(int lk, const double* boys_table, const BraTable& bra,                 \
                                        const KetTable& ket, const BatchMap& map, int total_items, double omega, \
                                        double* out, int* counter, cudaStream_t s);
#define EIP_DECL(I, J)                                                                                      \
    EIP_DECL_V(I, J, 0) EIP_DECL_V(I, J, 1) EIP_DECL_V(I, J, 2) EIP_DECL_V(I, J, 3) EIP_DECL_V(I, J, 4)     \
    EIP_DECL_V(I, J, 5) EIP_DECL_V(I, J, 6)                                                                 \
    EIP_DECL_F(I, J, 0) EIP_DECL_F(I, J, 2) EIP_DECL_F(I, J, 3) EIP_DECL_F(I, J, 4)                          \
    int launch_e_table_##I##J(const BraTable& bra, double* prim_E, cudaStream_t s);
EIP_DECL(0, 0) EIP_DECL(0, 1) EIP_DECL(1, 1) EIP_DECL(0, 2) EIP_DECL(1, 2) EIP_DECL(2, 2) EIP_DECL(0, 3) EIP_DECL(0, 4)
#undef EIP_DECL
#undef EIP_DECL_V
#undef EIP_DECL_F

// Fast pair classes: l_i <= l_j <= 2 (orbital shell pairs) and (0, 3), (0, 4)
// (a one-centre bra: the two-centre metric (P|Q) as pair class (0, l_P) with
// A = B = P).  Variant per (l_i, l_j, l_k), default 0; the autotuner's choices
// on B200 (tuning/b200_fp64.json) are applied with eip_tune_set.
static int g_variant[5][5][5] = {};
constexpr int kVariantsHost = 7;  // FP64 launch variants compiled (k3c_fast.cuh: kVariants)
// FP32 (mixed-precision) kernels: compiled variants 0, 2, 3, 4; default 0.
static int g_variant32[5][5][5] = {};

bool fast3c_supported(int li, int lj, int lk) {
    const bool pair_ok = li >= 0 && li <= lj && (lj <= 2 || (li == 0 && lj <= 4));
    return pair_ok && lk >= 0 && lk <= 4;
}

int fast3c_variant(int li, int lj, int lk) {
    return fast3c_supported(li, lj, lk) ? g_variant[li][lj][lk] : -1;
}

int fast3c_set_variant(int li, int lj, int lk, int v) {
    if (!fast3c_supported(li, lj, lk) || v < 0 || v >= kVariantsHost) return 1;
    g_variant[li][lj][lk] = v;
    return 0;
}

int fast3c_variant_fp32(int li, int lj, int lk) {
    return fast3c_supported(li, lj, lk) ? g_variant32[li][lj][lk] : -1;
}

int fast3c_set_variant_fp32(int li, int lj, int lk, int v) {
    if (!fast3c_supported(li, lj, lk) || !(v == 0 || v == 2 || v == 3 || v == 4)) return 1;
    g_variant32[li][lj][lk] = v;
    return 0;
}

// Doubles of one primitive pair's E record (e_record<li, lj>() in k3c_fast.cuh):
// E^{0 b}_t, b <= l_i + l_j (l_i > 0, l_j >= 2 only), then E^{i j}_t, for x, y and z.
size_t e_table_doubles(int li, int lj) {
    size_t n = 0;
    for (int i = 0; i <= li; i++)
        for (int j = 0; j <= lj; j++) n += i + j + 1;
    const size_t h = li > 0 && lj >= 2 ? (size_t)(li + lj + 1) * (li + lj + 2) / 2 : 0;
    return 3 * (n + h);
}

int launch_fast3c(int li, int lj, int lk, const BraTable& bra, const KetTable& ket, const BatchMap& map,
                  int total_items, double omega, double* out, int* counter, cudaStream_t s, bool fp32) {
    if (!fast3c_supported(li, lj, lk)) return 1;
    const double* t = boys_table_device();
    if (!t) return 2;
    const int v = fp32 ? -1 - g_variant32[li][lj][lk] : g_variant[li][lj][lk];
#define EIP_GO_V(I, J, V) return launch_fast3c_##I##J##_v##V(lk, t, bra, ket, map, total_items, omega, out, counter, s)
#define EIP_GO(I, J)                                                                                          \
    switch (v) {                                                                                              \
        case 1: EIP_GO_V(I, J, 1);                                                                            \
        case 2: EIP_GO_V(I, J, 2);                                                                            \
        case 3: EIP_GO_V(I, J, 3);                                                                            \
        case 4: EIP_GO_V(I, J, 4);                                                                            \
        case 5: EIP_GO_V(I, J, 5);                                                                            \
        case 6: EIP_GO_V(I, J, 6);                                                                            \
        case -1: return launch_fast3c_##I##J##_f32_v0(lk, t, bra, ket, map, total_items, omega, out, counter, s); \
        case -3: return launch_fast3c_##I##J##_f32_v2(lk, t, bra, ket, map, total_items, omega, out, counter, s); \
        case -4: return launch_fast3c_##I##J##_f32_v3(lk, t, bra, ket, map, total_items, omega, out, counter, s); \
        case -5: return launch_fast3c_##I##J##_f32_v4(lk, t, bra, ket, map, total_items, omega, out, counter, s); \
        default: EIP_GO_V(I, J, 0);                                                                           \
    }
    switch (li * 10 + lj) {
        case 0: EIP_GO(0, 0);
        case 1: EIP_GO(0, 1);
        case 11: EIP_GO(1, 1);
        case 2: EIP_GO(0, 2);
        case 12: EIP_GO(1, 2);
        case 22: EIP_GO(2, 2);
        case 3: EIP_GO(0, 3);
        case 4: EIP_GO(0, 4);
    }
#undef EIP_GO
#undef EIP_GO_V
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
        case 3: return launch_e_table_03(bra, prim_E, s);
        case 4: return launch_e_table_04(bra, prim_E, s);
    }
    return 1;
}

}  // namespace eip
